// gdfv_adjoint.cu -- hand-written vector-Jacobian product of the residual,
// g = (dR/dU)^T w, for the Euler path (2D or 3D) with the ausmdv or hllc flux and for
// MHD with hlle and GLM cleaning (FP64), and the adjoints of the predictor-corrector
// step and of a rollout built on it.
//
// The residual (e4/fvcell.d:824-856) is R_c = (1/V) sum_faces +-A F_f, each face
// flux F_f a function of the four stencil states (e4/onedinterp.d:751-989 and
// e4/fluxcalc.d:477-651 or :653-820), each state a function of U through decode_conserved
// (e4/fvcell.d:586-822) or through a boundary condition (ghost cells).  The VJP
// runs in three kernels:
//   1. per cell: decode U -> primitive state P = (rho, v0, v1, v2, u, a);
//   2. per face: recompute reconstruction and flux from P, then the reverse
//      sweep; cotangents land on the stencil cells' P (atomics), through the
//      ghost-cell maps (mirror, copy, xOrder-1 extrapolation, exchange), and on
//      the fixed inflow states;
//   3. per cell: reverse of decode, gU = (dP/dU)^T gP.
// Non-smooth points (limiter, clipping, fmax, Mach-number and upwind switches,
// the entropy fix, |.|) take the branch the primal values took; |x| has
// derivative +1 at x = 0 as in src/ntypes/complex.d:944-955.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/gdfv.h"
#include "gdfv_internal.h"
#include "gdfv_launch.h"

namespace gdfv {

namespace {

constexpr int NP = 6;  // rho, v0, v1, v2, u, a
constexpr int SRC_DONE = -1;  // a stencil source whose cotangent has been added already

__device__ __forceinline__ double sgn(double x) { return x < 0.0 ? -1.0 : 1.0; }

// Reciprocal for the adjoint arithmetic: a float estimate refined by two FP64
// Newton steps (relative error ~1e-14); exact division outside the float range.
__device__ __forceinline__ double rcp(double x) {
    double ax = fabs(x);
    if (!(ax > 1.0e-30 && ax < 1.0e30)) return 1.0 / x;
    double r = (double)__frcp_rn((float)x);
    r = r * (2.0 - x * r);
    r = r * (2.0 - x * r);
    return r;
}

// Reverse of clip_to_limits(q, A, B) (src/nm/limiters.d:41-50): routes g to q, A or B.
__device__ __forceinline__ void clip_rev(double q, double A, double B, double g, double& gq, double& gA, double& gB) {
    bool lowerIsA = A <= B;
    double lower = lowerIsA ? A : B;
    bool upperIsA = A > B;
    double upper = upperIsA ? A : B;
    double qc = (q > lower) ? q : lower;
    bool fromq = q > lower;
    if (qc <= upper) {
        if (fromq) gq += g;
        else if (lowerIsA) gA += g;
        else gB += g;
    } else {
        if (upperIsA) gA += g;
        else gB += g;
    }
}

// l2r2 for one scalar with equal lengths (e4/onedinterp.d:357-386), forward and reverse.
struct L2R2Rec {
    double dLm, del, dRp, sL, sR, nL, dL, nR, dR, X, Y, qLr, qRr;
    int eps_from;   // van_albada_variant lmr: epsilon from |q0| (1), |r0| (2) or the floor (0)
};

// LMR: the context may take van_albada_variant lmr (a face kernel with the rare rules)
template <bool LMR>
__device__ __forceinline__ void l2r2_fwd(const double* w, const NumParams& P, double q1, double q0, double r0,
                                         double r1, double& qL, double& qR, L2R2Rec& t) {
    t.dLm = (q0 - q1) * w[W_TOL];
    t.del = (r0 - q0) * w[W_TOC];
    t.dRp = (r1 - r0) * w[W_TOR];
    t.sL = 1.0; t.sR = 1.0;
    double eps = P.eps_van_albada;
    t.eps_from = 0;
    if (LMR && P.lmr_epsilon) {
        // lmr/onedinterp.d:147-151: the face's epsilon scaled by the larger of its two
        // states (both limiter values of the face take it), as the forward kernels form it
        const double tiny = 1e-12, a0 = fabs(q0), a1 = fabs(r0);
        const double m = fmax(fmax(tiny, a0), fmax(tiny, a1));
        t.eps_from = m == tiny ? 0 : (a0 >= a1 ? 1 : 2);
        eps = m * eps * w[W_TOC];
    }
    if (P.apply_limiter) {
        double pl = t.dLm * t.del, pr = t.del * t.dRp;
        t.nL = pl + fabs(pl) + eps; t.dL = t.dLm * t.dLm + t.del * t.del + eps; t.sL = t.nL * rcp(t.dL);
        t.nR = pr + fabs(pr) + eps; t.dR = t.del * t.del + t.dRp * t.dRp + eps; t.sR = t.nR * rcp(t.dR);
    }
    t.X = t.del * w[W_TWOL] + t.dLm * w[W_LENR0];
    t.Y = t.dRp * w[W_LENL0] + t.del * w[W_TWOR];
    t.qLr = q0 + t.sL * w[W_AL0] * t.X;
    t.qRr = r0 - t.sR * w[W_AR0] * t.Y;
    qL = t.qLr; qR = t.qRr;
    if (P.extrema_clipping) {
        qL = clip_to_limits(qL, q0, r0);
        qR = clip_to_limits(qR, q0, r0);
    }
}

template <bool LMR>
__device__ __forceinline__ void l2r2_rev(const double* w, const NumParams& P, double q1, double q0, double r0,
                                         double r1, const L2R2Rec& t, double gqL, double gqR, double& g1,
                                         double& g0, double& h0, double& h1) {
    double gqLr = 0.0, gqRr = 0.0;
    if (P.extrema_clipping) {
        clip_rev(t.qLr, q0, r0, gqL, gqLr, g0, h0);
        clip_rev(t.qRr, q0, r0, gqR, gqRr, g0, h0);
    } else {
        gqLr = gqL; gqRr = gqR;
    }
    double gdLm = 0.0, gdel = 0.0, gdRp = 0.0;
    // qLr = q0 + sL*aL0*X
    g0 += gqLr;
    double gsL = gqLr * w[W_AL0] * t.X;
    double gX = gqLr * t.sL * w[W_AL0];
    gdel += gX * w[W_TWOL];
    gdLm += gX * w[W_LENR0];
    // qRr = r0 - sR*aR0*Y
    h0 += gqRr;
    double gsR = -gqRr * w[W_AR0] * t.Y;
    double gY = -gqRr * t.sR * w[W_AR0];
    gdRp += gY * w[W_LENL0];
    gdel += gY * w[W_TWOR];
    if (P.apply_limiter) {
        // sL = nL/dL, nL = p + |p| + eps with p = dLm*del, dL = dLm^2 + del^2 + eps
        const double idL = rcp(t.dL);
        double gnL = gsL * idL, gdL = -gsL * t.sL * idL;
        double pl = t.dLm * t.del;
        double gpl = gnL * (1.0 + sgn(pl));
        gdLm += gpl * t.del + gdL * 2.0 * t.dLm;
        gdel += gpl * t.dLm + gdL * 2.0 * t.del;
        const double idR = rcp(t.dR);
        double gnR = gsR * idR, gdR = -gsR * t.sR * idR;
        double pr = t.del * t.dRp;
        double gpr = gnR * (1.0 + sgn(pr));
        gdel += gpr * t.dRp + gdR * 2.0 * t.del;
        gdRp += gpr * t.del + gdR * 2.0 * t.dRp;
        if (LMR && t.eps_from) {   // lmr: epsilon enters nL, dL, nR and dR
            const double geps = gnL + gdL + gnR + gdR;
            const double d = geps * P.eps_van_albada * w[W_TOC];
            if (t.eps_from == 1) g0 += d * sgn(q0);
            else h0 += d * sgn(r0);
        }
    }
    g0 += gdLm * w[W_TOL]; g1 -= gdLm * w[W_TOL];
    h0 += gdel * w[W_TOC]; g0 -= gdel * w[W_TOC];
    h1 += gdRp * w[W_TOR]; h0 -= gdRp * w[W_TOR];
}

// l2r2 on a graded block (recon_cell_graded's arithmetic): the left state of the face is
// cell L's plus-face value with L's weights gL[GW_*], the right state cell R's minus-face
// value with R's weights gR (e4/onedinterp.d:338-386 with each cell's own lengths); the
// difference across the face is scaled by L's and by R's weight separately.
struct L2R2G {
    double dLm, delL, delR, dRp, sL, sR, dL, dR, X, Y, qLr, qRr;
};

__device__ __forceinline__ void l2r2g_fwd(const double* gL, const double* gR, const NumParams& P, double q1,
                                          double q0, double r0, double r1, double& qL, double& qR, L2R2G& t) {
    t.dLm = (q0 - q1) * gL[GW_TOL];
    t.delL = (r0 - q0) * gL[GW_TOC];
    t.delR = (r0 - q0) * gR[GW_TOL];
    t.dRp = (r1 - r0) * gR[GW_TOC];
    t.sL = 1.0; t.sR = 1.0;
    const double eps = P.eps_van_albada;
    if (P.apply_limiter) {
        const double pl = t.dLm * t.delL, pr = t.delR * t.dRp;
        t.dL = t.dLm * t.dLm + t.delL * t.delL + eps; t.sL = (pl + fabs(pl) + eps) * rcp(t.dL);
        t.dR = t.delR * t.delR + t.dRp * t.dRp + eps; t.sR = (pr + fabs(pr) + eps) * rcp(t.dR);
    }
    t.X = t.delL * gL[GW_TWOL] + t.dLm * gL[GW_LENR0];
    t.Y = t.dRp * gR[GW_LENL0] + t.delR * gR[GW_TWOR];
    t.qLr = q0 + t.sL * gL[GW_A] * t.X;
    t.qRr = r0 - t.sR * gR[GW_A] * t.Y;
    qL = t.qLr; qR = t.qRr;
    if (P.extrema_clipping) {
        qL = clip_to_limits(qL, q0, r0);
        qR = clip_to_limits(qR, q0, r0);
    }
}

__device__ __forceinline__ void l2r2g_rev(const double* gL, const double* gR, const NumParams& P, double q0, double r0,
                                          const L2R2G& t, double gqL, double gqR, double& g1, double& g0, double& h0,
                                          double& h1) {
    double gqLr = 0.0, gqRr = 0.0;
    if (P.extrema_clipping) {
        clip_rev(t.qLr, q0, r0, gqL, gqLr, g0, h0);
        clip_rev(t.qRr, q0, r0, gqR, gqRr, g0, h0);
    } else {
        gqLr = gqL; gqRr = gqR;
    }
    double gdLm = 0.0, gdelL = 0.0, gdelR = 0.0, gdRp = 0.0;
    g0 += gqLr;
    const double gsL = gqLr * gL[GW_A] * t.X;
    const double gX = gqLr * t.sL * gL[GW_A];
    gdelL += gX * gL[GW_TWOL];
    gdLm += gX * gL[GW_LENR0];
    h0 += gqRr;
    const double gsR = -gqRr * gR[GW_A] * t.Y;
    const double gY = -gqRr * t.sR * gR[GW_A];
    gdRp += gY * gR[GW_LENL0];
    gdelR += gY * gR[GW_TWOR];
    if (P.apply_limiter) {
        // s = (p + |p| + eps) / d with p the product of the two differences, d their squares + eps
        const double idL = rcp(t.dL), idR = rcp(t.dR);
        const double gnL = gsL * idL, gdL = -gsL * t.sL * idL;
        const double pl = t.dLm * t.delL;
        const double gpl = gnL * (1.0 + sgn(pl));
        gdLm += gpl * t.delL + gdL * 2.0 * t.dLm;
        gdelL += gpl * t.dLm + gdL * 2.0 * t.delL;
        const double gnR = gsR * idR, gdR = -gsR * t.sR * idR;
        const double pr = t.delR * t.dRp;
        const double gpr = gnR * (1.0 + sgn(pr));
        gdelR += gpr * t.dRp + gdR * 2.0 * t.delR;
        gdRp += gpr * t.delR + gdR * 2.0 * t.dRp;
    }
    g0 += gdLm * gL[GW_TOL]; g1 -= gdLm * gL[GW_TOL];
    h0 += gdelL * gL[GW_TOC]; g0 -= gdelL * gL[GW_TOC];
    h0 += gdelR * gR[GW_TOL]; g0 -= gdelR * gR[GW_TOL];
    h1 += gdRp * gR[GW_TOC]; h0 -= gdRp * gR[GW_TOC];
}

// ausmdv (e4/fluxcalc.d:477-651) forward with the quantities the reverse needs,
// then its reverse.  Face-local states: r, p, u (normal), v, w (tangential), e, a.
struct FS { double r, p, u, v, w, e, a; };

__device__ void ausmdv_vjp(const NumParams& P, const FS& L, const FS& R, const double* gF, FS& gL, FS& gR) {
    // ---- forward
    const double irL = rcp(L.r), irR = rcp(R.r);
    double pLrL = L.p * irL, pRrR = R.p * irR;
    double keL = 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w);
    double keR = 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w);
    double HL = L.e + pLrL + keL, HR = R.e + pRrR + keR;
    double S = pLrL + pRrR;
    const double iS = rcp(S);
    double alphaL = 2.0 * pLrL * iS, alphaR = 2.0 * pRrR * iS;
    bool amL = L.a >= R.a;
    double am = fmax(L.a, R.a);
    const double iam = rcp(am);
    double ML = L.u * iam, MR = R.u * iam;
    double duL = 0.5 * (L.u + fabs(L.u));
    bool subL = fabs(ML) <= 1.0;
    double QL = (L.u + am) * (L.u + am) * (0.25 * iam);
    // p_half enters F linearly: only the cotangents of pLplus and pRminus are needed
    const double uLplus = subL ? alphaL * (QL - duL) + duL : duL;
    double duR = 0.5 * (R.u - fabs(R.u));
    bool subR = fabs(MR) <= 1.0;
    double QR = -(R.u - am) * (R.u - am) * (0.25 * iam);
    const double uRminus = subR ? alphaR * (QR - duR) + duR : duR;
    double ru_half = uLplus * L.r + uRminus * R.r;
    double dp0 = L.p - R.p;
    bool minL = L.p <= R.p;
    double mp = fmin(L.p, R.p);
    const double imp = rcp(mp);
    double dpa = 10.0 * fabs(dp0) * imp;
    bool sLin = dpa < 1.0;
    double s = 0.5 * fmin(1.0, dpa);
    double ru2V = uLplus * L.r * L.u + uRminus * R.r * R.u;
    double ru2D = 0.5 * (ru_half * (L.u + R.u) - fabs(ru_half) * (R.u - L.u));
    bool upL = ru_half >= 0.0;
    const double C = 0.125;
    bool caseA = ((L.u - L.a) < 0.0) && ((R.u - R.a) > 0.0);
    bool caseB = ((L.u + L.a) < 0.0) && ((R.u + R.a) > 0.0);
    double d_ua = 0.0;
    int efix = 0;
    if (P.apply_entropy_fix) {
        if (caseA && !caseB) { d_ua = C * ((R.u - R.a) - (L.u - L.a)); efix = 1; }
        if (caseB && !caseA) { d_ua = C * ((R.u + R.a) - (L.u + L.a)); efix = 2; }
    }
    // ---- reverse
    double gr_L = 0, gp_L = 0, gu_L = 0, gv_L = 0, gw_L = 0, ge_L = 0, ga_L = 0;
    double gr_R = 0, gp_R = 0, gu_R = 0, gv_R = 0, gw_R = 0, ge_R = 0, ga_R = 0;
    double gHL = 0, gHR = 0;
    if (efix && d_ua != 0.0) {
        double gd = -(gF[MASS] * (R.r - L.r) + gF[XMOM] * (R.r * R.u - L.r * L.u) + gF[YMOM] * (R.r * R.v - L.r * L.v) +
                      gF[ZMOM] * (R.r * R.w - L.r * L.w) + gF[TOTENERGY] * (R.r * HR - L.r * HL));
        gr_R -= gF[MASS] * d_ua; gr_L += gF[MASS] * d_ua;
        gr_R -= gF[XMOM] * d_ua * R.u; gu_R -= gF[XMOM] * d_ua * R.r; gr_L += gF[XMOM] * d_ua * L.u; gu_L += gF[XMOM] * d_ua * L.r;
        gr_R -= gF[YMOM] * d_ua * R.v; gv_R -= gF[YMOM] * d_ua * R.r; gr_L += gF[YMOM] * d_ua * L.v; gv_L += gF[YMOM] * d_ua * L.r;
        gr_R -= gF[ZMOM] * d_ua * R.w; gw_R -= gF[ZMOM] * d_ua * R.r; gr_L += gF[ZMOM] * d_ua * L.w; gw_L += gF[ZMOM] * d_ua * L.r;
        gr_R -= gF[TOTENERGY] * d_ua * HR; gHR -= gF[TOTENERGY] * d_ua * R.r;
        gr_L += gF[TOTENERGY] * d_ua * HL; gHL += gF[TOTENERGY] * d_ua * L.r;
        if (efix == 1) { gu_R += C * gd; ga_R -= C * gd; gu_L -= C * gd; ga_L += C * gd; }
        else { gu_R += C * gd; ga_R += C * gd; gu_L -= C * gd; ga_L -= C * gd; }
    }
    double vup = upL ? L.v : R.v, wup = upL ? L.w : R.w, Hup = upL ? HL : HR;
    double g_ru_half = gF[MASS] + gF[YMOM] * vup + gF[ZMOM] * wup + gF[TOTENERGY] * Hup;
    if (upL) { gv_L += gF[YMOM] * ru_half; gw_L += gF[ZMOM] * ru_half; gHL += gF[TOTENERGY] * ru_half; }
    else { gv_R += gF[YMOM] * ru_half; gw_R += gF[ZMOM] * ru_half; gHR += gF[TOTENERGY] * ru_half; }
    double g_ru2 = gF[XMOM], g_p_half = gF[XMOM];
    // ru2 = (0.5+s) ru2V + (0.5-s) ru2D
    double g_s = g_ru2 * (ru2V - ru2D);
    double g_ru2V = g_ru2 * (0.5 + s), g_ru2D = g_ru2 * (0.5 - s);
    // ru2D = 0.5 (ru_half (uL+uR) - |ru_half| (uR-uL))
    g_ru_half += 0.5 * g_ru2D * ((L.u + R.u) - sgn(ru_half) * (R.u - L.u));
    gu_L += 0.5 * g_ru2D * (ru_half + fabs(ru_half));
    gu_R += 0.5 * g_ru2D * (ru_half - fabs(ru_half));
    // ru2V = uLplus rL uL + uRminus rR uR
    double g_uLplus = g_ru2V * L.r * L.u, g_uRminus = g_ru2V * R.r * R.u;
    gr_L += g_ru2V * uLplus * L.u; gu_L += g_ru2V * uLplus * L.r;
    gr_R += g_ru2V * uRminus * R.u; gu_R += g_ru2V * uRminus * R.r;
    // s = 0.5 min(1, dpa), dpa = 10 |dp0| / min(pL, pR)
    if (sLin) {
        double g_dpa = 0.5 * g_s;
        double g_dp0 = g_dpa * 10.0 * sgn(dp0) * imp;
        double g_mp = -g_dpa * dpa * imp;
        gp_L += g_dp0; gp_R -= g_dp0;
        if (minL) gp_L += g_mp; else gp_R += g_mp;
    }
    double g_pLplus = g_p_half, g_pRminus = g_p_half;
    // ru_half = uLplus rL + uRminus rR
    g_uLplus += g_ru_half * L.r; gr_L += g_ru_half * uLplus;
    g_uRminus += g_ru_half * R.r; gr_R += g_ru_half * uRminus;
    double g_am = 0.0, g_alphaL = 0.0, g_alphaR = 0.0, g_duL = 0.0, g_duR = 0.0, g_ML = 0.0, g_MR = 0.0;
    if (subL) {
        gp_L += g_pLplus * (ML + 1.0) * (ML + 1.0) * (2.0 - ML) * 0.25;
        g_ML += g_pLplus * L.p * 0.25 * (2.0 * (ML + 1.0) * (2.0 - ML) - (ML + 1.0) * (ML + 1.0));
        g_alphaL += g_uLplus * (QL - duL);
        double g_Q = g_uLplus * alphaL;
        g_duL += g_uLplus * (1.0 - alphaL);
        gu_L += g_Q * 2.0 * (L.u + am) * (0.25 * iam);
        g_am += g_Q * ((L.u + am) * (0.5 * iam) - QL * iam);
    } else {
        const double iuL = rcp(L.u);
        gp_L += g_pLplus * duL * iuL;
        g_duL += g_pLplus * L.p * iuL;
        gu_L -= g_pLplus * L.p * duL * iuL * iuL;
        g_duL += g_uLplus;
    }
    gu_L += g_duL * 0.5 * (1.0 + sgn(L.u));
    if (subR) {
        gp_R += g_pRminus * (MR - 1.0) * (MR - 1.0) * (2.0 + MR) * 0.25;
        g_MR += g_pRminus * R.p * 0.25 * (2.0 * (MR - 1.0) * (2.0 + MR) + (MR - 1.0) * (MR - 1.0));
        g_alphaR += g_uRminus * (QR - duR);
        double g_Q = g_uRminus * alphaR;
        g_duR += g_uRminus * (1.0 - alphaR);
        gu_R += g_Q * (-2.0 * (R.u - am) * (0.25 * iam));
        g_am += g_Q * ((R.u - am) * (0.5 * iam) - QR * iam);
    } else {
        const double iuR = rcp(R.u);
        gp_R += g_pRminus * duR * iuR;
        g_duR += g_pRminus * R.p * iuR;
        gu_R -= g_pRminus * R.p * duR * iuR * iuR;
        g_duR += g_uRminus;
    }
    gu_R += g_duR * 0.5 * (1.0 - sgn(R.u));
    // ML = uL/am, MR = uR/am
    gu_L += g_ML * iam; g_am -= g_ML * ML * iam;
    gu_R += g_MR * iam; g_am -= g_MR * MR * iam;
    if (amL) ga_L += g_am; else ga_R += g_am;
    // alpha = 2 p/r / S
    double g_pLrL = g_alphaL * 2.0 * iS, g_pRrR = g_alphaR * 2.0 * iS;
    double g_S = -(g_alphaL * alphaL + g_alphaR * alphaR) * iS;
    g_pLrL += g_S; g_pRrR += g_S;
    // H = e + p/r + ke
    ge_L += gHL; g_pLrL += gHL; gu_L += gHL * L.u; gv_L += gHL * L.v; gw_L += gHL * L.w;
    ge_R += gHR; g_pRrR += gHR; gu_R += gHR * R.u; gv_R += gHR * R.v; gw_R += gHR * R.w;
    gp_L += g_pLrL * irL; gr_L -= g_pLrL * pLrL * irL;
    gp_R += g_pRrR * irR; gr_R -= g_pRrR * pRrR * irR;
    gL = FS{gr_L, gp_L, gu_L, gv_L, gw_L, ge_L, ga_L};
    gR = FS{gr_R, gp_R, gu_R, gv_R, gw_R, ge_R, ga_R};
}

// hllc (e4/fluxcalc.d:653-820, factor 1, one gas) forward with the quantities the reverse
// needs, then its reverse.  The Roe-averaged ratio of specific heats is gamma itself for
// one gas (its derivative vanishes); the wave-speed min/max and the star/side switches
// take the branches the primal values took.
__device__ void hllc_vjp(const NumParams& P, const FS& L, const FS& R, const double* gF, FS& gL, FS& gR) {
    // ---- forward
    const double g = P.gas.gamma;
    const double keL = 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w);
    const double keR = 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w);
    const double EL = L.r * L.e + L.r * keL, ER = R.r * R.e + R.r * keR;
    const double srL = sqrt(L.r), srR = sqrt(R.r);
    const double D = srL + srR, iD = rcp(D);
    const double uhat = (srL * L.u + srR * R.u) * iD;
    const double ghat = (srL * g + srR * g) * iD;
    const double N1 = srL * L.a * L.a + srR * R.a * R.a;
    const double sD = sqrt(D);
    const double T = D / sD;
    const double du = R.u - L.u;
    const double c2 = 0.5 * (ghat - 1.0);
    const double ahat2 = N1 * iD + c2 * T * du * du;
    const double ahat = sqrt(ahat2);
    const bool SLfromL = fmin(L.u - L.a, uhat - ahat) == L.u - L.a;
    const double SL = fmin(L.u - L.a, uhat - ahat);
    const bool SRfromR = fmax(R.u + R.a, uhat + ahat) == R.u + R.a;
    const double SR = fmax(R.u + R.a, uhat + ahat);
    const double num = R.p - L.p + L.r * L.u * (SL - L.u) - R.r * R.u * (SR - R.u);
    const double den = L.r * (SL - L.u) - R.r * (SR - R.u);
    const double iden = rcp(den);
    const double Ss = num * iden;
    const bool left = Ss > 0.0;
    const FS& X = left ? L : R;
    const double E = left ? EL : ER, S = left ? SL : SR;
    const bool star = left ? !(SL > 0.0) : !(SR < 0.0);
    const double dn = S - Ss, idn = star ? rcp(dn) : 0.0;
    const double coeff = star ? X.r * (S - X.u) * idn : 0.0;
    // ---- reverse (cotangents of the chosen side's r, p, u, v, w, E, S; of coeff, S*)
    double gr = 0, gp = 0, gu = 0, gv = 0, gw = 0, gE = 0, gS = 0, gc = 0, gSs = 0;
    // mass: r u (+ S (coeff - r))
    gr += gF[MASS] * X.u; gu += gF[MASS] * X.r;
    // momentum: r u u + p, r u v, r u w (+ S (coeff S* - r u), S (coeff - r) v, S (coeff - r) w)
    gr += gF[XMOM] * X.u * X.u; gu += gF[XMOM] * 2.0 * X.r * X.u; gp += gF[XMOM];
    gr += gF[YMOM] * X.u * X.v; gu += gF[YMOM] * X.r * X.v; gv += gF[YMOM] * X.r * X.u;
    gr += gF[ZMOM] * X.u * X.w; gu += gF[ZMOM] * X.r * X.w; gw += gF[ZMOM] * X.r * X.u;
    // energy: u (E + p) (+ S (U* - E))
    gu += gF[TOTENERGY] * (E + X.p); gE += gF[TOTENERGY] * X.u; gp += gF[TOTENERGY] * X.u;
    if (star) {
        gS += gF[MASS] * (coeff - X.r); gc += gF[MASS] * S; gr -= gF[MASS] * S;
        gS += gF[XMOM] * (coeff * Ss - X.r * X.u); gc += gF[XMOM] * S * Ss; gSs += gF[XMOM] * S * coeff;
        gr -= gF[XMOM] * S * X.u; gu -= gF[XMOM] * S * X.r;
        gS += gF[YMOM] * (coeff - X.r) * X.v; gc += gF[YMOM] * S * X.v; gr -= gF[YMOM] * S * X.v;
        gv += gF[YMOM] * S * (coeff - X.r);
        gS += gF[ZMOM] * (coeff - X.r) * X.w; gc += gF[ZMOM] * S * X.w; gr -= gF[ZMOM] * S * X.w;
        gw += gF[ZMOM] * S * (coeff - X.r);
        // U* = coeff (E/r + (S* - u) (S* + p/(r (S - u))))
        const double ir = rcp(X.r), Su = S - X.u, iSu = rcp(Su);
        const double Z = X.p * ir * iSu;
        const double Bq = Ss - X.u, Cq = Ss + Z;
        const double Xs = E * ir + Bq * Cq;
        const double Ust = coeff * Xs;
        gS += gF[TOTENERGY] * (Ust - E);
        gE -= gF[TOTENERGY] * S;
        const double gU = gF[TOTENERGY] * S;
        gc += gU * Xs;
        const double gX = gU * coeff;
        gE += gX * ir; gr -= gX * E * ir * ir;
        gSs += gX * Cq; gu -= gX * Cq;
        const double gZ = gX * Bq;
        gSs += gZ;
        gp += gZ * ir * iSu; gr -= gZ * Z * ir;
        const double gSu = -gZ * Z * iSu;
        gS += gSu; gu -= gSu;
        // coeff = r (S - u) / (S - S*)
        gr += gc * Su * idn;
        gS += gc * X.r * idn; gu -= gc * X.r * idn;
        const double gdn = -gc * coeff * idn;
        gS += gdn; gSs -= gdn;
    }
    // E = r e + r ke on the chosen side
    const double ke = left ? keL : keR;
    gr += gE * (X.e + ke);
    double ge = gE * X.r;
    gu += gE * X.r * X.u; gv += gE * X.r * X.v; gw += gE * X.r * X.w;
    double gr_L = 0, gp_L = 0, gu_L = 0, gv_L = 0, gw_L = 0, ge_L = 0, ga_L = 0;
    double gr_R = 0, gp_R = 0, gu_R = 0, gv_R = 0, gw_R = 0, ge_R = 0, ga_R = 0;
    double gSL = 0, gSR = 0;
    if (left) { gr_L += gr; gp_L += gp; gu_L += gu; gv_L += gv; gw_L += gw; ge_L += ge; gSL += gS; }
    else { gr_R += gr; gp_R += gp; gu_R += gu; gv_R += gv; gw_R += gw; ge_R += ge; gSR += gS; }
    // S* = num / den
    const double gnum = gSs * iden, gden = -gSs * Ss * iden;
    gp_R += gnum; gp_L -= gnum;
    gr_L += gnum * L.u * (SL - L.u); gu_L += gnum * L.r * (SL - 2.0 * L.u); gSL += gnum * L.r * L.u;
    gr_R -= gnum * R.u * (SR - R.u); gu_R -= gnum * R.r * (SR - 2.0 * R.u); gSR -= gnum * R.r * R.u;
    gr_L += gden * (SL - L.u); gSL += gden * L.r; gu_L -= gden * L.r;
    gr_R -= gden * (SR - R.u); gSR -= gden * R.r; gu_R += gden * R.r;
    // SL = min(uL - aL, uhat - ahat), SR = max(uR + aR, uhat + ahat)
    double guhat = 0.0, gahat = 0.0;
    if (SLfromL) { gu_L += gSL; ga_L -= gSL; } else { guhat += gSL; gahat -= gSL; }
    if (SRfromR) { gu_R += gSR; ga_R += gSR; } else { guhat += gSR; gahat += gSR; }
    // ahat2 = N1 / D + c2 T du^2, T = D / sqrt(D); ahat = sqrt(ahat2)
    const double gah2 = gahat * 0.5 / ahat;
    const double gN1 = gah2 * iD;
    double gD = -gah2 * N1 * iD * iD;
    double gsrL = gN1 * L.a * L.a, gsrR = gN1 * R.a * R.a;
    ga_L += gN1 * 2.0 * srL * L.a; ga_R += gN1 * 2.0 * srR * R.a;
    gD += gah2 * c2 * du * du * 0.5 / sD;
    const double gdu = gah2 * c2 * T * 2.0 * du;
    gu_R += gdu; gu_L -= gdu;
    // uhat = (srL uL + srR uR) / D
    gsrL += guhat * L.u * iD; gu_L += guhat * srL * iD;
    gsrR += guhat * R.u * iD; gu_R += guhat * srR * iD;
    gD -= guhat * uhat * iD;
    gsrL += gD; gsrR += gD;
    gr_L += gsrL * 0.5 / srL; gr_R += gsrR * 0.5 / srR;
    gL = FS{gr_L, gp_L, gu_L, gv_L, gw_L, ge_L, ga_L};
    gR = FS{gr_R, gp_R, gu_R, gv_R, gw_R, ge_R, ga_R};
}

// Reverse of the simple outflow flux of cell state q (rho, v0, v1, v2, u, a) through a
// face of normal +axis D (simple_outflow_flux, boundary_flux_effect.d:504-645): F = the
// cell's convective flux plus p n when the mass flux leaves (outsign m > 0), else p n
// alone; g the cotangent of the global-frame flux, added into gq.
template <int D>
__device__ void simple_flux_vjp(const NumParams& P, const double* q, int outsign, const double* g, double* gq) {
    const double rho = q[0], u = q[4];
    const double v[3] = {q[1], q[2], q[3]};
    const double T = u * P.gas.Cvinv;
    const double p = rho * P.gas.R * T;
    const double vn = v[D];
    const double m = rho * vn;
    double gp = 0.0, gm = 0.0, gvn = 0.0, gu = 0.0;
    double gv[3] = {0.0, 0.0, 0.0};
    if (outsign * m > 0.0) {
        gm += g[MASS];
        for (int d = 0; d < 3; ++d) {
            if (d == 2 && P.dims != 3) continue;   // no z momentum flux in 2D
            const double gd = g[XMOM + d];
            if (d == D) gp += gd;
            gv[d] += gd * m;
            gm += gd * v[d];
        }
        const double utot = u + 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        gm += g[TOTENERGY] * utot;
        gu += g[TOTENERGY] * m;
        for (int d = 0; d < 3; ++d) gv[d] += g[TOTENERGY] * m * v[d];
        gp += g[TOTENERGY] * vn;
        gvn += g[TOTENERGY] * p;
    } else {
        gp += g[XMOM + D];
    }
    gq[0] += gm * vn;                     // m = rho vn
    gvn += gm * rho;
    gv[D] += gvn;
    gq[0] += gp * P.gas.R * T;            // p = rho R (u Cvinv)
    gu += gp * rho * P.gas.R * P.gas.Cvinv;
    gq[1] += gv[0];
    gq[2] += gv[1];
    gq[3] += gv[2];
    gq[4] += gu;
}

// hlle for ideal MHD (e4/fluxcalc.d:1608-1780, mu0 = 1) forward with the quantities the
// reverse needs, then its reverse.  Face-local states: r, p, u (normal), v, w
// (tangential), B (normal, tangential, tangential), e (internal energy).  The
// alpha-weighted Cv and R of one gas are Cv and R themselves (their derivatives vanish);
// the wave-speed min/max and the switches at 0 take the branches the primal values took;
// SAFESQRT's floor (|x| <= 1e-14: 0) has derivative 0.
struct FSm { double r, p, u, v, w, Bx, By, Bz, e; };

struct FastSpeed {   // cf = sqrt(0.5 (alf + sqrt(alf^2 - 4 a2 ca2))) with its pieces
    double a2, ca2, alf, X, als, cf2, cf;
    bool live;        // SAFESQRT took the root
};
__device__ __forceinline__ FastSpeed fast_speed(double gam, double p, double rho, double Bx, double By, double Bz) {
    FastSpeed f;
    const double BB = Bx * Bx + By * By + Bz * Bz;
    f.a2 = gam * p / rho;
    f.ca2 = Bx * Bx / rho;
    f.alf = f.a2 + BB / rho;
    f.X = f.alf * f.alf - 4.0 * f.a2 * f.ca2;
    f.live = fabs(f.X) > 1.0e-14;
    f.als = f.live ? sqrt(f.X) : 0.0;
    f.cf2 = 0.5 * (f.alf + f.als);
    f.cf = sqrt(f.cf2);
    return f;
}
// reverse of fast_speed: gcf into the cotangents of p, rho and B (added)
__device__ __forceinline__ void fast_speed_rev(const FastSpeed& f, double gam, double p, double rho, double Bx,
                                               double By, double Bz, double gcf, double& gp, double& grho,
                                               double& gBx, double& gBy, double& gBz) {
    const double gcf2 = gcf * 0.5 / f.cf;
    double galf = 0.5 * gcf2, gals = 0.5 * gcf2;
    double ga2 = 0.0, gca2 = 0.0;
    if (f.live) {
        const double gX = gals * 0.5 / f.als;
        galf += gX * 2.0 * f.alf;
        ga2 += -4.0 * f.ca2 * gX;
        gca2 += -4.0 * f.a2 * gX;
    }
    const double BB = Bx * Bx + By * By + Bz * Bz;
    // alf = a2 + BB / rho
    ga2 += galf;
    const double gBB = galf / rho;
    grho -= galf * BB / (rho * rho);
    // ca2 = Bx^2 / rho
    double gBx2 = gca2 / rho;
    grho -= gca2 * f.ca2 / rho;
    // a2 = gam p / rho
    gp += ga2 * gam / rho;
    grho -= ga2 * f.a2 / rho;
    gBx2 += gBB;
    gBx += 2.0 * Bx * gBx2;
    gBy += 2.0 * By * gBB;
    gBz += 2.0 * Bz * gBB;
}

// The one-sided fluxes of hlle_mhd: mass, x, y, z momentum, energy, By, Bz (Bx: 0).
__device__ __forceinline__ void mhd_side_flux(const FSm& S, double* f) {
    const double BB = S.Bx * S.Bx + S.By * S.By + S.Bz * S.Bz;
    const double pt = S.p + 0.5 * BB;
    const double uu = S.u * S.u + S.v * S.v + S.w * S.w;
    f[0] = S.r * S.u;
    f[1] = S.r * S.u * S.u - S.Bx * S.Bx + pt;
    f[2] = S.r * S.u * S.v - S.Bx * S.By;
    f[3] = S.r * S.u * S.w - S.Bx * S.Bz;
    f[4] = (S.r * S.e + 0.5 * (S.r * uu + BB) + pt) * S.u - (S.u * S.Bx + S.v * S.By + S.w * S.Bz) * S.Bx;
    f[5] = S.u * S.By - S.v * S.Bx;
    f[6] = S.u * S.Bz - S.w * S.Bx;
}
// reverse of mhd_side_flux: cotangents gf[7] into gS (added)
__device__ __forceinline__ void mhd_side_flux_rev(const FSm& S, const double* gf, FSm& gS) {
    const double BB = S.Bx * S.Bx + S.By * S.By + S.Bz * S.Bz;
    const double pt = S.p + 0.5 * BB;
    const double uu = S.u * S.u + S.v * S.v + S.w * S.w;
    double gpt = 0.0, guu = 0.0, gBB = 0.0;
    // mass
    gS.r += gf[0] * S.u; gS.u += gf[0] * S.r;
    // x momentum r u^2 - Bx^2 + pt
    gS.r += gf[1] * S.u * S.u; gS.u += gf[1] * 2.0 * S.r * S.u; gS.Bx -= gf[1] * 2.0 * S.Bx; gpt += gf[1];
    // y, z momentum
    gS.r += gf[2] * S.u * S.v; gS.u += gf[2] * S.r * S.v; gS.v += gf[2] * S.r * S.u;
    gS.Bx -= gf[2] * S.By; gS.By -= gf[2] * S.Bx;
    gS.r += gf[3] * S.u * S.w; gS.u += gf[3] * S.r * S.w; gS.w += gf[3] * S.r * S.u;
    gS.Bx -= gf[3] * S.Bz; gS.Bz -= gf[3] * S.Bx;
    // energy (H) u - (u Bx + v By + w Bz) Bx, H = r e + (r uu + BB)/2 + pt
    const double H = S.r * S.e + 0.5 * (S.r * uu + BB) + pt;
    const double Sd = S.u * S.Bx + S.v * S.By + S.w * S.Bz;
    const double gH = gf[4] * S.u;
    gS.u += gf[4] * H;
    const double gSd = -gf[4] * S.Bx;
    gS.Bx -= gf[4] * Sd;
    gS.r += gH * (S.e + 0.5 * uu); gS.e += gH * S.r; guu += 0.5 * gH * S.r; gBB += 0.5 * gH; gpt += gH;
    gS.u += gSd * S.Bx; gS.Bx += gSd * S.u; gS.v += gSd * S.By; gS.By += gSd * S.v;
    gS.w += gSd * S.Bz; gS.Bz += gSd * S.w;
    // By, Bz induction
    gS.u += gf[5] * S.By; gS.By += gf[5] * S.u; gS.v -= gf[5] * S.Bx; gS.Bx -= gf[5] * S.v;
    gS.u += gf[6] * S.Bz; gS.Bz += gf[6] * S.u; gS.w -= gf[6] * S.Bx; gS.Bx -= gf[6] * S.w;
    // pt = p + BB/2, uu, BB
    gS.p += gpt; gBB += 0.5 * gpt;
    gS.u += 2.0 * S.u * guu; gS.v += 2.0 * S.v * guu; gS.w += 2.0 * S.w * guu;
    gS.Bx += 2.0 * S.Bx * gBB; gS.By += 2.0 * S.By * gBB; gS.Bz += 2.0 * S.Bz * gBB;
}

// gF: cotangent of the face-local flux in the order MASS, XMOM, YMOM, ZMOM, TOTENERGY, XB,
// YB, ZB; gL, gR receive the cotangents of the two states (added).
__device__ void hlle_mhd_vjp(const NumParams& P, const FSm& L, const FSm& R, const double* gF, FSm& gL, FSm& gR) {
    // ---- forward
    const double gam = (P.gas.Cv + P.gas.R) / P.gas.Cv;
    const double rho = 0.5 * (L.r + R.r), p = 0.5 * (L.p + R.p), u = 0.5 * (L.u + R.u);
    const double Bx = 0.5 * (L.Bx + R.Bx), By = 0.5 * (L.By + R.By), Bz = 0.5 * (L.Bz + R.Bz);
    const FastSpeed fm = fast_speed(gam, p, rho, Bx, By, Bz);
    const FastSpeed fL = fast_speed(gam, L.p, L.r, L.Bx, L.By, L.Bz);
    const FastSpeed fR = fast_speed(gam, R.p, R.r, R.Bx, R.By, R.Bz);
    const double wp = u + fm.cf, wm = u - fm.cf, wmL = L.u - fL.cf, wpR = R.u + fR.cf;
    const bool blL = wmL <= wm, brR = wpR >= wp;
    const double bl = blL ? wmL : wm, br = brR ? wpR : wp;
    const double blm = fmin(bl, 0.0), brp = fmax(br, 0.0);
    double fl[7], fr[7];
    mhd_side_flux(L, fl);
    mhd_side_flux(R, fr);
    const double uuL = L.u * L.u + L.v * L.v + L.w * L.w, uuR = R.u * R.u + R.v * R.v + R.w * R.w;
    const double BBL = L.Bx * L.Bx + L.By * L.By + L.Bz * L.Bz, BBR = R.Bx * R.Bx + R.By * R.By + R.Bz * R.Bz;
    // one-sided fluxes and jumps in the order of F (the Bx flux of either side is 0)
    const double fLF[8] = {fl[0], fl[1], fl[2], fl[3], fl[4], 0.0, fl[5], fl[6]};
    const double fRF[8] = {fr[0], fr[1], fr[2], fr[3], fr[4], 0.0, fr[5], fr[6]};
    const double d[8] = {R.r - L.r, R.r * R.u - L.r * L.u, R.r * R.v - L.r * L.v, R.r * R.w - L.r * L.w,
                         (R.p - L.p) / (gam - 1.0) + 0.5 * (R.r * uuR + BBR) - 0.5 * (L.r * uuL + BBL),
                         R.Bx - L.Bx, R.By - L.By, R.Bz - L.Bz};
    const double iden = 1.0 / (brp - blm), fac1 = brp * blm;
    // ---- reverse
    double gbrp = 0.0, gblm = 0.0, gfac1 = 0.0, giden = 0.0;
    double gfLF[8], gfRF[8], gd[8];
    for (int q = 0; q < 8; ++q) {
        const double N = brp * fLF[q] - blm * fRF[q] + fac1 * d[q];
        const double gN = gF[q] * iden;
        giden += gF[q] * N;
        gfLF[q] = gN * brp;
        gfRF[q] = -gN * blm;
        gd[q] = gN * fac1;
        gbrp += gN * fLF[q];
        gblm -= gN * fRF[q];
        gfac1 += gN * d[q];
    }
    gbrp += -giden * iden * iden;
    gblm += giden * iden * iden;
    gbrp += gfac1 * blm;
    gblm += gfac1 * brp;
    // fmin(bl, 0), fmax(br, 0) keep their first argument on a tie (src/ntypes/complex.d)
    const double gbl = bl <= 0.0 ? gblm : 0.0, gbr = br >= 0.0 ? gbrp : 0.0;
    double gwm = 0.0, gwp = 0.0, gcfL = 0.0, gcfR = 0.0;
    if (blL) { gL.u += gbl; gcfL -= gbl; } else gwm += gbl;
    if (brR) { gR.u += gbr; gcfR += gbr; } else gwp += gbr;
    // wp = u + cf, wm = u - cf of the averages
    const double gu = gwp + gwm, gcf = gwp - gwm;
    double gp = 0.0, grho = 0.0, gBx = 0.0, gBy = 0.0, gBz = 0.0;
    fast_speed_rev(fm, gam, p, rho, Bx, By, Bz, gcf, gp, grho, gBx, gBy, gBz);
    fast_speed_rev(fL, gam, L.p, L.r, L.Bx, L.By, L.Bz, gcfL, gL.p, gL.r, gL.Bx, gL.By, gL.Bz);
    fast_speed_rev(fR, gam, R.p, R.r, R.Bx, R.By, R.Bz, gcfR, gR.p, gR.r, gR.Bx, gR.By, gR.Bz);
    gL.r += 0.5 * grho; gR.r += 0.5 * grho;
    gL.p += 0.5 * gp; gR.p += 0.5 * gp;
    gL.u += 0.5 * gu; gR.u += 0.5 * gu;
    gL.Bx += 0.5 * gBx; gR.Bx += 0.5 * gBx;
    gL.By += 0.5 * gBy; gR.By += 0.5 * gBy;
    gL.Bz += 0.5 * gBz; gR.Bz += 0.5 * gBz;
    const double gfl[7] = {gfLF[0], gfLF[1], gfLF[2], gfLF[3], gfLF[4], gfLF[6], gfLF[7]};
    const double gfr[7] = {gfRF[0], gfRF[1], gfRF[2], gfRF[3], gfRF[4], gfRF[6], gfRF[7]};
    mhd_side_flux_rev(L, gfl, gL);
    mhd_side_flux_rev(R, gfr, gR);
    // jumps
    gR.r += gd[0]; gL.r -= gd[0];
    gR.r += gd[1] * R.u; gR.u += gd[1] * R.r; gL.r -= gd[1] * L.u; gL.u -= gd[1] * L.r;
    gR.r += gd[2] * R.v; gR.v += gd[2] * R.r; gL.r -= gd[2] * L.v; gL.v -= gd[2] * L.r;
    gR.r += gd[3] * R.w; gR.w += gd[3] * R.r; gL.r -= gd[3] * L.w; gL.w -= gd[3] * L.r;
    const double ig = gd[4] / (gam - 1.0);
    gR.p += ig; gL.p -= ig;
    gR.r += 0.5 * gd[4] * uuR; gL.r -= 0.5 * gd[4] * uuL;
    gR.u += gd[4] * R.r * R.u; gR.v += gd[4] * R.r * R.v; gR.w += gd[4] * R.r * R.w;
    gL.u -= gd[4] * L.r * L.u; gL.v -= gd[4] * L.r * L.v; gL.w -= gd[4] * L.r * L.w;
    gR.Bx += gd[4] * R.Bx; gR.By += gd[4] * R.By; gR.Bz += gd[4] * R.Bz;
    gL.Bx -= gd[4] * L.Bx; gL.By -= gd[4] * L.By; gL.Bz -= gd[4] * L.Bz;
    gR.Bx += gd[5]; gL.Bx -= gd[5];
    gR.By += gd[6]; gL.By -= gd[6];
    gR.Bz += gd[7]; gL.Bz -= gd[7];
}

struct AdjArgs {
    const BlockDesc* blocks;
    const InflowState* inflow;
    const double* U;
    const double* W;
    double* Pp;        // [6][total]
    double* gP;        // [6][total]
    double* gU;        // [nq][total]
    double* gInflow;   // [ninflow][6]
    const double* rot; // rotations of exchange faces with an Rmatrix (9 doubles each)
    const long long* face_off;  // [3][nblocks+1] prefix counts of faces per direction
    double* lam;       // [nq][total] adjoint state of a fused step (modes 1, 2)
    double* bbuf;      // [nq][total] b = dt/2 lam + dt mu (mode 1 writes, mode 2 is its W)
    double w_scale;    // W enters scaled by this
    double dt;
    long long total;
    int nblocks;
    int mode;          // 0: gU = result; 1: mu -> bbuf, lam += mu; 2: lam += result
    NumParams P;
    double c_h;        // MHD: the GLM wave speed of the residual (the context's current one)
    // MHD with cleaning in a step adjoint: {c_h, psi damping factor} of the step (device;
    // null: c_h above, no damping); chd_slot is where the step adjoint forms them
    const double* chd;
    double* chd_slot;
};

__device__ __forceinline__ void decode_cell(const AdjArgs& a, long long g) {
    double u[5];
    for (int q = 0; q < 5; ++q) u[q] = a.U[q * a.total + g];
    Prim<double> s;
    double p, T;
    decode(a.P, u, s, p, T);
    double v[NP] = {s.rho, s.v[0], s.v[1], s.v[2], s.u, s.a};
    for (int m = 0; m < NP; ++m) { a.Pp[m * a.total + g] = v[m]; a.gP[m * a.total + g] = 0.0; }
}

__global__ void adj_decode_kernel(AdjArgs a) {
    long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g < a.total) decode_cell(a, g);
}

// Stencil cell state from P (with the ghost maps) and the reverse map of a cotangent.
struct Src {
    const BlockDesc* blk;
    long long c0, c1;
    int kind, axis, inflow;
};

// RARE: some exchange rotates its ghosts' vectors, some face is an outflow boundary
// with a ghost or flux rule of its own, the limiter is lmr's, or some block is graded
// (the face kernels without it carry none of that code)
template <bool RARE>
__device__ Src adj_resolve(const AdjArgs& a, const BlockDesc& B, int i, int j, int k) {
    StageArgs A{};
    A.blocks = a.blocks;
    CellSrc s = resolve<RARE, RARE>(A, B, i, j, k);
    return Src{s.blk, s.c0, s.c1, s.kind, s.axis, s.inflow};
}

template <bool RARE>
__device__ void adj_load(const AdjArgs& a, const Src& s, double* c) {
    if (s.kind == SRC_INFLOW) {
        const InflowState& in = a.inflow[s.inflow];
        c[0] = in.rho; c[1] = in.vel[0]; c[2] = in.vel[1]; c[3] = in.vel[2]; c[4] = in.u; c[5] = in.a;
        return;
    }
    const long long g0 = s.blk->offset + s.c0;
    double e[NP];
    for (int m = 0; m < NP; ++m) e[m] = a.Pp[m * a.total + g0];
    if (s.kind == SRC_EXTRAP1_G0 || s.kind == SRC_EXTRAP1_G1) {
        const long long g1 = s.blk->offset + s.c1;
        double f[NP];
        for (int m = 0; m < NP; ++m) f[m] = a.Pp[m * a.total + g1];
        // ghost0 = 2e - f1, ghost1 = 2 ghost0 - e (rho, v, u); a from the edge cell
        for (int m = 0; m < 5; ++m) {
            double g0v = 2.0 * e[m] - f[m];
            c[m] = (s.kind == SRC_EXTRAP1_G0) ? g0v : 2.0 * g0v - e[m];
        }
        c[5] = e[5];
        return;
    }
    for (int m = 0; m < NP; ++m) c[m] = e[m];
    if (s.kind == SRC_MIRROR) c[1 + s.axis] = -c[1 + s.axis];
    if (RARE && s.kind == SRC_ROTATE) {   // ghost velocity R v (flowstate.d:393-400)
        const double* R = a.rot + 9 * s.inflow;
        for (int r = 0; r < 3; ++r) c[1 + r] = R[3 * r] * e[1] + R[3 * r + 1] * e[2] + R[3 * r + 2] * e[3];
    }
    if (RARE && s.kind == SRC_FIXEDP) {   // fixed_p.d:98-119: rho, u from p_outside at the cell's T
        const double T = e[4] * a.P.gas.Cvinv;
        c[0] = a.inflow[s.inflow].p / (T * a.P.gas.R);
        c[4] = a.P.gas.Cv * T;
    }
    if (RARE && s.kind == SRC_FIXEDPT) {  // fixed_pt.d:105-128: rho, u from p_outside, T_outside
        c[0] = a.inflow[s.inflow].rho;
        c[4] = a.inflow[s.inflow].u;
    }
}

template <bool RARE>
__device__ void adj_scatter(const AdjArgs& a, const Src& s, const double* gc) {
    if (s.kind == SRC_INFLOW) {
        for (int m = 0; m < NP; ++m) atomicAdd(&a.gInflow[s.inflow * NP + m], gc[m]);
        return;
    }
    const long long g0 = s.blk->offset + s.c0;
    if (s.kind == SRC_EXTRAP1_G0 || s.kind == SRC_EXTRAP1_G1) {
        const long long g1 = s.blk->offset + s.c1;
        const double ce = (s.kind == SRC_EXTRAP1_G0) ? 2.0 : 3.0, cf = (s.kind == SRC_EXTRAP1_G0) ? -1.0 : -2.0;
        for (int m = 0; m < 5; ++m) {
            atomicAdd(&a.gP[m * a.total + g0], ce * gc[m]);
            atomicAdd(&a.gP[m * a.total + g1], cf * gc[m]);
        }
        atomicAdd(&a.gP[5 * a.total + g0], gc[5]);
        return;
    }
    if (RARE && (s.kind == SRC_FIXEDP || s.kind == SRC_FIXEDPT)) {
        // velocity and sound speed pass through; rho and u are the outside state's
        // (FixedPT) or, FixedP, rho = p/(T R) and u = Cv T with T = u_cell / Cv
        double gu = 0.0;
        if (s.kind == SRC_FIXEDP) {
            const double u = a.Pp[4 * a.total + g0];
            const double T = u * a.P.gas.Cvinv;
            const double rho = a.inflow[s.inflow].p / (T * a.P.gas.R);
            gu = gc[0] * (-rho / T) * a.P.gas.Cvinv + gc[4] * a.P.gas.Cv * a.P.gas.Cvinv;
        }
        atomicAdd(&a.gP[1 * a.total + g0], gc[1]);
        atomicAdd(&a.gP[2 * a.total + g0], gc[2]);
        atomicAdd(&a.gP[3 * a.total + g0], gc[3]);
        if (gu != 0.0) atomicAdd(&a.gP[4 * a.total + g0], gu);
        atomicAdd(&a.gP[5 * a.total + g0], gc[5]);
        return;
    }
    if (RARE && s.kind == SRC_ROTATE) {   // the transpose of the ghost's rotation R v
        const double* R = a.rot + 9 * s.inflow;
        for (int m = 0; m < NP; ++m) {
            const double v = (m >= 1 && m <= 3)
                                 ? R[m - 1] * gc[1] + R[3 + m - 1] * gc[2] + R[6 + m - 1] * gc[3]
                                 : gc[m];
            atomicAdd(&a.gP[m * a.total + g0], v);
        }
        return;
    }
    for (int m = 0; m < NP; ++m) {
        double v = gc[m];
        if (s.kind == SRC_MIRROR && m == 1 + s.axis) v = -v;
        atomicAdd(&a.gP[m * a.total + g0], v);
    }
}

// ---------------------------------------------------------------- MHD (residual VJP)
// Primitives of an MHD cell: rho, v0, v1, v2, u, a, B0, B1, B2, psi.
constexpr int NPM = 10;

// Stencil state of an MHD source (the ghost rules of finish_cell): (x, y) is the centre
// of the stencil cell, for the slip wall's dipole field (internal_copy_then_reflect.d:
// 140-143: Bx, By of a slip-wall ghost with |x| < 0.4136 are the dipole's, constants).
__device__ void adj_load_mhd(const AdjArgs& a, const Src& s, double x, double y, double* c) {
    if (s.kind == SRC_INFLOW) {
        const InflowState& in = a.inflow[s.inflow];
        c[0] = in.rho; c[1] = in.vel[0]; c[2] = in.vel[1]; c[3] = in.vel[2]; c[4] = in.u; c[5] = in.a;
        c[6] = in.B[0]; c[7] = in.B[1]; c[8] = in.B[2]; c[9] = in.psi;
        return;
    }
    const long long g0 = s.blk->offset + s.c0;
    double e[NPM];
    for (int m = 0; m < NPM; ++m) e[m] = a.Pp[m * a.total + g0];
    for (int m = 0; m < NPM; ++m) c[m] = e[m];
    if (s.kind == SRC_EXTRAP1_G0 || s.kind == SRC_EXTRAP1_G1) {
        // extrapolate_copy.d:171-201: rho, u, v, B extrapolated; a and psi of the edge cell
        const long long g1 = s.blk->offset + s.c1;
        for (int m = 0; m < NPM; ++m) {
            if (m == 5 || m == 9) continue;
            const double f = a.Pp[m * a.total + g1];
            const double g0v = 2.0 * e[m] - f;
            c[m] = (s.kind == SRC_EXTRAP1_G0) ? g0v : 2.0 * g0v - e[m];
        }
    } else if (s.kind == SRC_MIRROR) {
        c[1 + s.axis] = -c[1 + s.axis];   // B is not reflected (ghost_cell.d:56-67)
        if (x > -0.4136 && x < 0.4136) dipole_field(x, y, c[6], c[7]);
    } else if (s.kind == SRC_ROTATE) {
        const double* R = a.rot + 9 * s.inflow;
        for (int r = 0; r < 3; ++r) {
            c[1 + r] = R[3 * r] * e[1] + R[3 * r + 1] * e[2] + R[3 * r + 2] * e[3];
            c[6 + r] = R[3 * r] * e[6] + R[3 * r + 1] * e[7] + R[3 * r + 2] * e[8];
        }
    }
}

__device__ void adj_scatter_mhd(const AdjArgs& a, const Src& s, double x, double y, const double* gc) {
    if (s.kind == SRC_INFLOW) {
        for (int m = 0; m < NPM; ++m) atomicAdd(&a.gInflow[s.inflow * NPM + m], gc[m]);
        return;
    }
    const long long g0 = s.blk->offset + s.c0;
    if (s.kind == SRC_EXTRAP1_G0 || s.kind == SRC_EXTRAP1_G1) {
        const long long g1 = s.blk->offset + s.c1;
        const double ce = (s.kind == SRC_EXTRAP1_G0) ? 2.0 : 3.0, cf = (s.kind == SRC_EXTRAP1_G0) ? -1.0 : -2.0;
        for (int m = 0; m < NPM; ++m) {
            if (m == 5 || m == 9) { atomicAdd(&a.gP[m * a.total + g0], gc[m]); continue; }
            atomicAdd(&a.gP[m * a.total + g0], ce * gc[m]);
            atomicAdd(&a.gP[m * a.total + g1], cf * gc[m]);
        }
        return;
    }
    double g[NPM];
    for (int m = 0; m < NPM; ++m) g[m] = gc[m];
    if (s.kind == SRC_MIRROR) {
        g[1 + s.axis] = -g[1 + s.axis];
        if (x > -0.4136 && x < 0.4136) { g[6] = 0.0; g[7] = 0.0; }   // the dipole's constants
    } else if (s.kind == SRC_ROTATE) {
        const double* R = a.rot + 9 * s.inflow;
        for (int m = 0; m < 3; ++m) {
            g[1 + m] = R[m] * gc[1] + R[3 + m] * gc[2] + R[6 + m] * gc[3];
            g[6 + m] = R[m] * gc[6] + R[3 + m] * gc[7] + R[6 + m] * gc[8];
        }
    }
    for (int m = 0; m < NPM; ++m) atomicAdd(&a.gP[m * a.total + g0], g[m]);
}

// Block and cell indices of face f of direction D (the face lies between cells
// index-1 and index along D).
template <int D>
__device__ __forceinline__ int face_coords(const AdjArgs& a, long long f, int& i, int& j, int& k) {
    const long long* off = a.face_off + D * (a.nblocks + 1);
    int b = 0;
    while (off[b + 1] <= f) ++b;
    const BlockDesc& B = a.blocks[b];
    // 32-bit: the host limits a block's faces of one direction to 2^31 - 1
    const unsigned lf = (unsigned)(f - off[b]);
    const unsigned nf0 = B.n[0] + (D == 0), nf1 = B.n[1] + (D == 1);
    const unsigned r = lf / nf0;
    i = (int)(lf - r * nf0);
    k = (int)(r / nf1);
    j = (int)(r - (unsigned)k * nf1);
    return b;
}

// Source of stencil cell m (index -2, -1, 0, +1 along D from the face).  A face
// whose four stencil cells lie inside its block (the other two indices always do)
// takes them directly; the boundary rules apply to the others.
template <int D, bool RARE>
__device__ __forceinline__ Src stencil_src(const AdjArgs& a, const BlockDesc& B, int i, int j, int k, int m) {
    const int idxD = D == 0 ? i : (D == 1 ? j : k);
    if (idxD >= 2 && idxD + 1 < B.n[D]) {
        const int sD = D == 0 ? 1 : (D == 1 ? B.n[0] : B.n[0] * B.n[1]);
        const int c = i + B.n[0] * (j + B.n[1] * k) + (m - 2) * sD;
        return Src{&B, (long long)c, -1, SRC_CELL, D, 0};
    }
    return adj_resolve<RARE>(a, B, i - (D == 0 ? 2 - m : 0), j - (D == 1 ? 2 - m : 0), k - (D == 2 ? 2 - m : 0));
}

// The reverse sweep of face f of direction D: cotangents gc[m] of the stencil
// cells (added to), the kind of each stencil source and the inflow state the
// stencil reaches (if any).  Only these small records stay live: the sources
// themselves are resolved again when the cotangents are scattered.
// rowid identifies the line of faces (block and the two other indices).
template <int D, int FLUX, bool RARE>
__device__ __forceinline__ void face_vjp(const AdjArgs& a, int b, int i, int j, int k, int* kind, int& inflow,
                                         double (*gc)[NP], long long& rowid) {
    const BlockDesc& B = a.blocks[b];
    rowid = (long long)b * 0x100000000ll + (D == 0 ? (long long)j + (long long)B.n[1] * k : (long long)i);
    double c[4][NP];
    for (int m = 0; m < 4; ++m) {
        const Src sm = stencil_src<D, RARE>(a, B, i, j, k, m);
        kind[m] = sm.kind;
        if (sm.kind == SRC_INFLOW) inflow = sm.inflow;
        adj_load<RARE>(a, sm, c[m]);
    }
    // cotangent of the face flux: F enters R_right with +A/V and R_left with -A/V
    const double AV = B.area[D] * B.vol_inv * a.w_scale;
    const int nD = B.n[D];
    const int idxD = D == 0 ? i : (D == 1 ? j : k);
    const bool leftIn = idxD - 1 >= 0, rightIn = idxD < nD;
    const long long gl = B.offset + (long long)(i - (D == 0)) + (long long)B.n[0] * ((long long)(j - (D == 1)) + (long long)B.n[1] * (k - (D == 2)));
    const long long gr = B.offset + (long long)i + (long long)B.n[0] * ((long long)j + (long long)B.n[1] * k);
    double AVr = AV, AVl = AV;
    bool graded = false;
    const double* gwL = nullptr;
    const double* gwR = nullptr;
    if constexpr (RARE) {
        if (B.graded) {
            // graded block: the face's area from the lengths of its cells across it, each
            // side's own volume (cell lengths glen[d][c + 2], weights of cells -1 .. n)
            graded = true;
            const int ic[3] = {i, j, k};
            double Lr[3], Ll[3];
            for (int d = 0; d < 3; ++d) {
                Lr[d] = B.glen[d][ic[d] + 2];
                Ll[d] = B.glen[d][ic[d] - (d == D) + 2];
            }
            const bool threeD = a.P.dims == 3;
            const double Af = threeD ? (D == 0 ? Lr[1] * Lr[2] : (D == 1 ? Lr[2] * Lr[0] : Lr[0] * Lr[1]))
                                     : (D == 0 ? Lr[1] : Lr[0]);
            const double Vr = threeD ? Lr[0] * Lr[1] * Lr[2] : Lr[0] * Lr[1];
            const double Vl = threeD ? Ll[0] * Ll[1] * Ll[2] : Ll[0] * Ll[1];
            AVr = Af / Vr * a.w_scale;
            AVl = Af / Vl * a.w_scale;
            gwL = B.gw[D] + (long long)idxD * GW_N;
            gwR = gwL + GW_N;
        }
    }
    double gFg[5];
    for (int q = 0; q < 5; ++q) {
        double wr = rightIn ? a.W[q * a.total + gr] : 0.0;
        double wl = leftIn ? a.W[q * a.total + gl] : 0.0;
        gFg[q] = AVr * wr - AVl * wl;
    }
    if constexpr (RARE) {
        // OutFlowBC_SimpleFlux (boundary_flux_effect.d:504-645): the boundary face's flux is
        // the interior cell's outflow flux, or only its pressure on a closed face
        const int bface = idxD == 0 ? 2 * D : (idxD == nD ? 2 * D + 1 : -1);
        if (bface >= 0 && B.bc_type[bface] == BC_SIMPLE_FLUX) {
            const int in = (bface & 1) ? 1 : 2;   // the interior cell: left of a plus face
            simple_flux_vjp<D>(a.P, c[in], (bface & 1) ? 1 : -1, gFg, gc[in]);
            return;
        }
    }
    constexpr int ax0 = D, ax1 = (D + 1) % 3, ax2 = (D + 2) % 3;
    double gF[5] = {gFg[MASS], gFg[XMOM + ax0], gFg[XMOM + ax1], gFg[XMOM + ax2], gFg[TOTENERGY]};
    // ---- forward reconstruction (local-frame scalars: vn, vt1, vt2, rho, u)
    const double* w = B.w[D];
    const NumParams& P = a.P;
    const int pv[5] = {1 + ax0, 1 + ax1, 1 + ax2, 0, 4};
    double qL[5], qR[5];
    for (int sc = 0; sc < 5; ++sc) {
        if (RARE && graded) {
            L2R2G rg;
            l2r2g_fwd(gwL, gwR, P, c[0][pv[sc]], c[1][pv[sc]], c[2][pv[sc]], c[3][pv[sc]], qL[sc], qR[sc], rg);
            continue;
        }
        L2R2Rec rec;  // recomputed in the reverse sweep rather than kept live
        l2r2_fwd<RARE>(w, P, c[0][pv[sc]], c[1][pv[sc]], c[2][pv[sc]], c[3][pv[sc]], qL[sc], qR[sc], rec);
    }
    const double Rg = P.gas.R, Cvinv = P.gas.Cvinv;
    bool badL = qL[4] <= 0.0 || qL[3] <= 0.0, badR = qR[4] <= 0.0 || qR[3] <= 0.0;
    FS L, Rs;
    if (badL) L = FS{c[1][0], c[1][0] * Rg * (c[1][4] * Cvinv), c[1][pv[0]], c[1][pv[1]], c[1][pv[2]], c[1][4], c[1][5]};
    else L = FS{qL[3], qL[3] * Rg * (qL[4] * Cvinv), qL[0], qL[1], qL[2], qL[4], c[1][5]};
    if (badR) Rs = FS{c[2][0], c[2][0] * Rg * (c[2][4] * Cvinv), c[2][pv[0]], c[2][pv[1]], c[2][pv[2]], c[2][4], c[2][5]};
    else Rs = FS{qR[3], qR[3] * Rg * (qR[4] * Cvinv), qR[0], qR[1], qR[2], qR[4], c[2][5]};
    // ---- reverse
    FS gL, gR;
    if constexpr (FLUX == FLUX_HLLC) hllc_vjp(P, L, Rs, gF, gL, gR);
    else ausmdv_vjp(P, L, Rs, gF, gL, gR);
    gc[1][5] += gL.a;
    gc[2][5] += gR.a;
    double gqL[5] = {0, 0, 0, 0, 0}, gqR[5] = {0, 0, 0, 0, 0};
    // p = rho R (u Cvinv)
    if (badL) {
        gc[1][0] += gL.r + gL.p * Rg * (c[1][4] * Cvinv);
        gc[1][4] += gL.e + gL.p * c[1][0] * Rg * Cvinv;
        gc[1][pv[0]] += gL.u; gc[1][pv[1]] += gL.v; gc[1][pv[2]] += gL.w;
    } else {
        gqL[3] += gL.r + gL.p * Rg * (qL[4] * Cvinv);
        gqL[4] += gL.e + gL.p * qL[3] * Rg * Cvinv;
        gqL[0] += gL.u; gqL[1] += gL.v; gqL[2] += gL.w;
    }
    if (badR) {
        gc[2][0] += gR.r + gR.p * Rg * (c[2][4] * Cvinv);
        gc[2][4] += gR.e + gR.p * c[2][0] * Rg * Cvinv;
        gc[2][pv[0]] += gR.u; gc[2][pv[1]] += gR.v; gc[2][pv[2]] += gR.w;
    } else {
        gqR[3] += gR.r + gR.p * Rg * (qR[4] * Cvinv);
        gqR[4] += gR.e + gR.p * qR[3] * Rg * Cvinv;
        gqR[0] += gR.u; gqR[1] += gR.v; gqR[2] += gR.w;
    }
    for (int sc = 0; sc < 5; ++sc) {
        const int v = pv[sc];
        if (RARE && graded) {
            L2R2G rg;
            double ql, qr;
            l2r2g_fwd(gwL, gwR, P, c[0][v], c[1][v], c[2][v], c[3][v], ql, qr, rg);
            l2r2g_rev(gwL, gwR, P, c[1][v], c[2][v], rg, gqL[sc], gqR[sc], gc[0][v], gc[1][v], gc[2][v], gc[3][v]);
            continue;
        }
        L2R2Rec rec;
        double ql, qr;
        l2r2_fwd<RARE>(w, P, c[0][v], c[1][v], c[2][v], c[3][v], ql, qr, rec);
        l2r2_rev<RARE>(w, P, c[0][v], c[1][v], c[2][v], c[3][v], rec, gqL[sc], gqR[sc], gc[0][v], gc[1][v], gc[2][v],
                 gc[3][v]);
    }
}

// Face f of direction D, one thread.  Along i (D = 0) the four faces whose
// stencils share a cell are neighbouring lanes of one warp: their contributions
// to that cell are summed with shuffles first, and one lane adds the sum
// (same-address atomics from one warp would serialise).
#ifndef GDFV_ADJ_MINB
#define GDFV_ADJ_MINB 3
#endif
template <int D, int FLUX, bool RARE>
__device__ __forceinline__ void face_thread(const AdjArgs& a, long long f) {
    const long long* off = a.face_off + D * (a.nblocks + 1);
    const bool act = f < off[a.nblocks];
    int kind[4] = {SRC_DONE, SRC_DONE, SRC_DONE, SRC_DONE};
    int inflow = -1;
    double gc[4][NP];
    for (int m = 0; m < 4; ++m)
        for (int q = 0; q < NP; ++q) gc[m][q] = 0.0;
    long long rowid = -1 - (long long)threadIdx.x;   // distinct for inactive lanes
    int b = 0, i = 0, j = 0, k = 0;
    if (act) {
        b = face_coords<D>(a, f, i, j, k);
        face_vjp<D, FLUX, RARE>(a, b, i, j, k, kind, inflow, gc, rowid);
    }
    if (D == 0) {
        const unsigned full = 0xffffffffu;
        const int lane = threadIdx.x & 31;
        // source lane l + d holds the contribution of its stencil cell m to the
        // cell of lane l (its own stencil cell 2): m = 0 at d = 2, m = 1 at d = 1, m = 3 at d = -1
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            const int m = t == 0 ? 0 : (t == 1 ? 1 : 3);
            const int d = t == 0 ? 2 : (t == 1 ? 1 : -1);
            const bool mine = act && kind[m] == SRC_CELL;
            const int from = lane + d, to = lane - d;
            const long long row_from = __shfl_sync(full, rowid, from & 31);
            const int ok_from = __shfl_sync(full, (int)mine, from & 31);
            const long long row_to = __shfl_sync(full, rowid, to & 31);
            const bool recv = from >= 0 && from < 32 && act && ok_from && row_from == rowid;
            const bool sent = to >= 0 && to < 32 && mine && row_to == rowid;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                const double v = __shfl_sync(full, gc[m][q], from & 31);
                if (recv) gc[2][q] += v;
                if (sent) gc[m][q] = 0.0;
            }
            if (sent) kind[m] = SRC_DONE;   // nothing left to scatter for this source
        }
    }
    // Inflow ghost states are shared by every face along an inflow boundary: sum the
    // warp's cotangents per inflow state (a face's stencil crosses at most one
    // boundary face, so a lane carries at most one state), one atomic per state.
    {
        const unsigned full = 0xffffffffu;
        int key = -1;
        double vin[NP];
#pragma unroll
        for (int q = 0; q < NP; ++q) vin[q] = 0.0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (act && kind[m] == SRC_INFLOW) {
                key = inflow;
#pragma unroll
                for (int q = 0; q < NP; ++q) vin[q] += gc[m][q];
                kind[m] = SRC_DONE;
            }
        }
        if (__ballot_sync(full, key >= 0)) {
            const unsigned grp = __match_any_sync(full, key);
            const int lane = threadIdx.x & 31;
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                double acc = 0.0;
                for (int src = 0; src < 32; ++src) {
                    const double v = __shfl_sync(full, vin[q], src);
                    if ((grp >> src) & 1u) acc += v;
                }
                vin[q] = acc;
            }
            if (key >= 0 && lane == __ffs(grp) - 1)
                for (int q = 0; q < NP; ++q) atomicAdd(&a.gInflow[key * NP + q], vin[q]);
        }
    }
    if (!act) return;
    const BlockDesc& B = a.blocks[b];
    for (int m = 0; m < 4; ++m)
        if (kind[m] >= 0) adj_scatter<RARE>(a, stencil_src<D, RARE>(a, B, i, j, k, m), gc[m]);
}

// All faces of the three directions in one launch: CTAs [0, nb0) take the i faces,
// [nb0, nb0 + nb1) the j faces, the rest the k faces (128 faces per CTA).
constexpr int FACE_CTA = 128;
template <int FLUX, bool RARE>
__global__ void __launch_bounds__(FACE_CTA, GDFV_ADJ_MINB) adj_faces_kernel(AdjArgs a, unsigned nb0, unsigned nb1) {
    const unsigned bid = blockIdx.x;
    if (bid < nb0) face_thread<0, FLUX, RARE>(a, (long long)bid * FACE_CTA + threadIdx.x);
    else if (bid < nb0 + nb1) face_thread<1, FLUX, RARE>(a, (long long)(bid - nb0) * FACE_CTA + threadIdx.x);
    else face_thread<2, FLUX, RARE>(a, (long long)(bid - nb0 - nb1) * FACE_CTA + threadIdx.x);
}

// The reverse sweep of MHD face f of direction D (face_flux with hlle_mhd and the GLM
// terms, e4/fluxcalc.d:54-187, :1608-1780): cotangents of the four stencil cells'
// primitives, scattered through the ghost rules.  The limiter's arithmetic is the Euler
// path's; psi is reconstructed only with divergence cleaning (a copy of the cell's
// otherwise); c_h is the residual's, frozen.
// Slot of primitive v in a face thread's shared-memory copy of its stencil: the sound
// speed (5) is never reconstructed, so the nine others are kept.
__device__ __forceinline__ constexpr int SL(int v) { return v < 5 ? v : v - 1; }
template <int D, bool RARE>
__device__ void face_mhd(const AdjArgs& a, long long f, double* smt) {
    const long long* off = a.face_off + D * (a.nblocks + 1);
    if (f >= off[a.nblocks]) return;
    int i = 0, j = 0, k = 0;
    const int b = face_coords<D>(a, f, i, j, k);
    const BlockDesc& B = a.blocks[b];
    const NumParams& P = a.P;
    Src src[4];
    double xs[4], ys[4];
    // the stencil's primitives and their cotangents in this thread's shared-memory slot
    double (*c)[9] = reinterpret_cast<double (*)[9]>(smt);
    double (*gc)[9] = reinterpret_cast<double (*)[9]>(smt + 4 * 9);
    for (int m = 0; m < 4; ++m) {
        src[m] = stencil_src<D, RARE>(a, B, i, j, k, m);
        const int ci = i - (D == 0 ? 2 - m : 0), cj = j - (D == 1 ? 2 - m : 0);
        xs[m] = B.x0 + ((double)ci + 0.5) * B.len[0];
        ys[m] = B.y0 + ((double)cj + 0.5) * B.len[1];
        double t[NPM];
        adj_load_mhd(a, src[m], xs[m], ys[m], t);
#pragma unroll
        for (int v = 0; v < NPM; ++v) if (v != 5) c[m][SL(v)] = t[v];
    }
    const double AV = B.area[D] * B.vol_inv * a.w_scale;
    const int nD = B.n[D];
    const int idxD = D == 0 ? i : (D == 1 ? j : k);
    const bool leftIn = idxD - 1 >= 0, rightIn = idxD < nD;
    const long long gl = B.offset + (long long)(i - (D == 0)) +
                         (long long)B.n[0] * ((long long)(j - (D == 1)) + (long long)B.n[1] * (k - (D == 2)));
    const long long gr = B.offset + (long long)i + (long long)B.n[0] * ((long long)j + (long long)B.n[1] * k);
    double gFg[10];
    for (int q = 0; q < 10; ++q) {
        const double wr = rightIn ? a.W[q * a.total + gr] : 0.0;
        const double wl = leftIn ? a.W[q * a.total + gl] : 0.0;
        gFg[q] = AV * (wr - wl);
    }
    constexpr int ax0 = D, ax1 = (D + 1) % 3, ax2 = (D + 2) % 3;
    double gF[10];
    gF[MASS] = gFg[MASS]; gF[TOTENERGY] = gFg[TOTENERGY]; gF[PSI] = gFg[PSI]; gF[DIVB] = gFg[DIVB];
    gF[XMOM] = gFg[XMOM + ax0]; gF[YMOM] = gFg[XMOM + ax1]; gF[ZMOM] = gFg[XMOM + ax2];
    gF[XB] = gFg[XB + ax0]; gF[YB] = gFg[XB + ax1]; gF[ZB] = gFg[XB + ax2];
    // ---- forward reconstruction: face-frame v, rho, u, face-frame B, psi
    const double* w = B.w[D];
    const int pv[9] = {1 + ax0, 1 + ax1, 1 + ax2, 0, 4, 6 + ax0, 6 + ax1, 6 + ax2, 9};
    const bool clean = P.divergence_cleaning;
    double qL[9], qR[9];
    for (int sc = 0; sc < 9; ++sc) {
        if (sc == 8 && !clean) { qL[8] = c[1][SL(9)]; qR[8] = c[2][SL(9)]; continue; }
        L2R2Rec rec;
        l2r2_fwd<true>(w, P, c[0][SL(pv[sc])], c[1][SL(pv[sc])], c[2][SL(pv[sc])], c[3][SL(pv[sc])], qL[sc], qR[sc], rec);
    }
    const double Rg = P.gas.R, Cvinv = P.gas.Cvinv;
    const bool badL = qL[4] <= 0.0 || qL[3] <= 0.0, badR = qR[4] <= 0.0 || qR[3] <= 0.0;
    auto state = [&](bool bad, const double* q, const double* cell, FSm& S, double& psi) {
        if (bad) {   // e4/onedinterp.d:44-74: the cell-centre state
            S = FSm{cell[SL(0)], cell[SL(0)] * Rg * (cell[SL(4)] * Cvinv), cell[SL(pv[0])], cell[SL(pv[1])], cell[SL(pv[2])],
                    cell[SL(pv[5])], cell[SL(pv[6])], cell[SL(pv[7])], cell[SL(4)]};
            psi = cell[SL(9)];
        } else {
            S = FSm{q[3], q[3] * Rg * (q[4] * Cvinv), q[0], q[1], q[2], q[5], q[6], q[7], q[4]};
            psi = q[8];
        }
    };
    FSm L, R;
    double psiL, psiR;
    state(badL, qL, c[1], L, psiL);
    state(badR, qR, c[2], R, psiR);
    // ---- reverse: F[divB] = (BxR - BxL)/2 and the GLM terms (fluxcalc.d:139-150, with the
    // reference's third term added to F[xB] under glm_reference_indexing)
    FSm gL{}, gR{};
    double gpsiL = 0.0, gpsiR = 0.0;
    gR.Bx += 0.5 * gF[DIVB]; gL.Bx -= 0.5 * gF[DIVB];
    if (clean) {
        const double ch = a.chd ? a.chd[0] : a.c_h;
        const double gt3 = P.glm_reference_indexing ? gF[XB] : gF[ZB];
        const double gpa = gF[XB] + gF[YB] + gt3;
        gR.Bx -= 0.5 * ch * gF[XB]; gL.Bx += 0.5 * ch * gF[XB];
        gR.By -= 0.5 * ch * gF[YB]; gL.By += 0.5 * ch * gF[YB];
        gR.Bz -= 0.5 * ch * gt3; gL.Bz += 0.5 * ch * gt3;
        gpsiL += 0.5 * gpa; gpsiR += 0.5 * gpa;
        const double gps = gF[PSI] * ch * ch;
        gL.Bx += 0.5 * gps; gR.Bx += 0.5 * gps;
        gpsiR -= gps / (2.0 * ch); gpsiL += gps / (2.0 * ch);
    }
    const double gF8[8] = {gF[MASS], gF[XMOM], gF[YMOM], gF[ZMOM], gF[TOTENERGY], gF[XB], gF[YB], gF[ZB]};
    hlle_mhd_vjp(P, L, R, gF8, gL, gR);
    for (int m = 0; m < 4; ++m)
        for (int q = 0; q < 9; ++q) gc[m][q] = 0.0;
    double gqL[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, gqR[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    auto back = [&](bool bad, const FSm& S, const FSm& gS, double gpsi, double* gq, double* gcell) {
        // p = rho R (u Cvinv)
        const double gr_ = gS.r + gS.p * Rg * (S.e * Cvinv), ge_ = gS.e + gS.p * S.r * Rg * Cvinv;
        if (bad) {
            gcell[SL(0)] += gr_; gcell[SL(4)] += ge_;
            gcell[SL(pv[0])] += gS.u; gcell[SL(pv[1])] += gS.v; gcell[SL(pv[2])] += gS.w;
            gcell[SL(pv[5])] += gS.Bx; gcell[SL(pv[6])] += gS.By; gcell[SL(pv[7])] += gS.Bz; gcell[SL(9)] += gpsi;
        } else {
            gq[3] += gr_; gq[4] += ge_;
            gq[0] += gS.u; gq[1] += gS.v; gq[2] += gS.w;
            gq[5] += gS.Bx; gq[6] += gS.By; gq[7] += gS.Bz; gq[8] += gpsi;
        }
    };
    back(badL, L, gL, gpsiL, gqL, gc[1]);
    back(badR, R, gR, gpsiR, gqR, gc[2]);
    for (int sc = 0; sc < 9; ++sc) {
        const int v = pv[sc];
        if (sc == 8 && !clean) { gc[1][SL(9)] += gqL[8]; gc[2][SL(9)] += gqR[8]; continue; }
        L2R2Rec rec;
        double ql, qr;
        l2r2_fwd<true>(w, P, c[0][SL(v)], c[1][SL(v)], c[2][SL(v)], c[3][SL(v)], ql, qr, rec);
        l2r2_rev<true>(w, P, c[0][SL(v)], c[1][SL(v)], c[2][SL(v)], c[3][SL(v)], rec, gqL[sc], gqR[sc], gc[0][SL(v)], gc[1][SL(v)], gc[2][SL(v)],
                       gc[3][SL(v)]);
    }
    for (int m = 0; m < 4; ++m) {
        double t[NPM];
#pragma unroll
        for (int v = 0; v < NPM; ++v) t[v] = v == 5 ? 0.0 : gc[m][SL(v)];
        adj_scatter_mhd(a, src[m], xs[m], ys[m], t);
    }
}

// RARE: some exchange rotates its ghosts' vectors (the only rare rule MHD takes).
// Each thread keeps its stencil's primitives and cotangents (nine of each per cell, 72
// doubles) in shared memory at a stride of 73 doubles (conflict-free for 8-byte
// accesses): 74.75 KB per CTA of 128 threads, 3 CTAs per SM at 168 registers, with the
// carveout that gives shared memory the most room.
constexpr int MHD_SLOT = 8 * 9 + 1;
constexpr size_t MHD_FACE_SMEM = sizeof(double) * MHD_SLOT * 128;
template <bool RARE>
__global__ void __launch_bounds__(128, 3) adj_faces_mhd_kernel(AdjArgs a, unsigned nb0, unsigned nb1) {
    extern __shared__ double smem_mhd[];
    double* smt = smem_mhd + threadIdx.x * MHD_SLOT;
    const unsigned bid = blockIdx.x;
    if (bid < nb0) face_mhd<0, RARE>(a, (long long)bid * 128 + threadIdx.x, smt);
    else if (bid < nb0 + nb1) face_mhd<1, RARE>(a, (long long)(bid - nb0) * 128 + threadIdx.x, smt);
    else face_mhd<2, RARE>(a, (long long)(bid - nb0 - nb1) * 128 + threadIdx.x, smt);
}

void launch_faces_mhd(const AdjArgs& a, const unsigned* nb, cudaStream_t s) {
    static bool attr_set[2] = {false, false};   // dynamic shared memory above 48 KB, once per instantiation
    // (the attributes are the function's, for the process's device)
    const int r = a.P.rotating ? 1 : 0;
    if (!attr_set[r]) {
        if (r) cudaFuncSetAttribute(adj_faces_mhd_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MHD_FACE_SMEM);
        else cudaFuncSetAttribute(adj_faces_mhd_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MHD_FACE_SMEM);
        if (r) cudaFuncSetAttribute(adj_faces_mhd_kernel<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        else cudaFuncSetAttribute(adj_faces_mhd_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        attr_set[r] = true;
    }
    const unsigned n = nb[0] + nb[1] + nb[2];
    if (r) adj_faces_mhd_kernel<true><<<n, 128, MHD_FACE_SMEM, s>>>(a, nb[0], nb[1]);
    else adj_faces_mhd_kernel<false><<<n, 128, MHD_FACE_SMEM, s>>>(a, nb[0], nb[1]);
}

// MHD decode (e4/fvcell.d:586-822): the ten primitives of each cell, gP cleared.
__device__ __forceinline__ void decode_cell_mhd(const AdjArgs& a, long long g) {
    double u[10];
    for (int q = 0; q < 10; ++q) u[q] = a.U[q * a.total + g];
    if (a.mode == 1 && a.chd) {
        // the corrector's stencils read the predictor state with psi damped, U1' = D U1
        // (D: psi times the step's damping factor), and its cotangent is D lam
        const double damp = a.chd[1];
        u[PSI] *= damp;
        a.lam[PSI * a.total + g] *= damp;
    }
    Prim<double> s;
    double p, T;
    decode(a.P, u, s, p, T);
    const double v[NPM] = {s.rho, s.v[0], s.v[1], s.v[2], s.u, s.a, s.B[0], s.B[1], s.B[2], s.psi};
    for (int m = 0; m < NPM; ++m) { a.Pp[m * a.total + g] = v[m]; a.gP[m * a.total + g] = 0.0; }
}

__global__ void adj_decode_mhd_kernel(AdjArgs a) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g < a.total) decode_cell_mhd(a, g);
}

// gU = (dP/dU)^T gP for the MHD decode: u = (E - |B|^2/2)/rho - |v|^2/2, B and psi
// copied, a = sqrt(gamma R u / Cv); divB does not enter the primitives.  The modes
// of back_cell (the predictor-corrector adjoint's lam and b updates) over ten
// conserved quantities.
__device__ __forceinline__ void back_cell_mhd(const AdjArgs& a, long long g) {
    double U[10], gp[NPM];
    for (int q = 0; q < 10; ++q) U[q] = a.U[q * a.total + g];
    for (int m = 0; m < NPM; ++m) gp[m] = a.gP[m * a.total + g];
    const double rho = U[MASS], dinv = 1.0 / rho;
    const double v0 = U[XMOM] * dinv, v1 = U[YMOM] * dinv, v2 = U[ZMOM] * dinv;
    const double rE = U[TOTENERGY] - 0.5 * (U[XB] * U[XB] + U[YB] * U[YB] + U[ZB] * U[ZB]);
    const double u = rE * dinv - 0.5 * (v0 * v0 + v1 * v1 + v2 * v2);
    const double gR = a.P.gas.gamma * a.P.gas.R;
    const double aa = sqrt(gR * u * a.P.gas.Cvinv);
    const double gu = gp[4] + gp[5] * gR * a.P.gas.Cvinv / (2.0 * aa);
    const double gv0 = gp[1] - gu * v0, gv1 = gp[2] - gu * v1, gv2 = gp[3] - gu * v2;
    const double gdinv = gu * rE + gv0 * U[XMOM] + gv1 * U[YMOM] + gv2 * U[ZMOM];
    double r[10];
    r[MASS] = gp[0] - gdinv * dinv * dinv;
    r[XMOM] = gv0 * dinv; r[YMOM] = gv1 * dinv; r[ZMOM] = gv2 * dinv;
    r[TOTENERGY] = gu * dinv;
    r[XB] = gp[6] - gu * dinv * U[XB];
    r[YB] = gp[7] - gu * dinv * U[YB];
    r[ZB] = gp[8] - gu * dinv * U[ZB];
    r[PSI] = gp[9];
    r[DIVB] = 0.0;
    if (a.mode == 0) {
        for (int q = 0; q < 10; ++q) a.gU[q * a.total + g] = r[q];
    } else if (a.mode == 1) {
        if (a.chd) r[PSI] *= a.chd[1];   // mu is the cotangent of U1' = D U1: D mu is U1's
        for (int q = 0; q < 10; ++q) {
            const double l = a.lam[q * a.total + g];
            a.bbuf[q * a.total + g] = 0.5 * a.dt * l + a.dt * r[q];
            a.lam[q * a.total + g] = l + r[q];
        }
    } else {
        for (int q = 0; q < 10; ++q) a.lam[q * a.total + g] += r[q];
    }
}

__global__ void adj_back_mhd_kernel(AdjArgs a) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g < a.total) back_cell_mhd(a, g);
}

__global__ void adj_back_decode_mhd_kernel(AdjArgs back, AdjArgs next) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= back.total) return;
    back_cell_mhd(back, g);
    decode_cell_mhd(next, g);
}

// gU = (dP/dU)^T gP for P = decode(U) (e4/fvcell.d:586-822 with ideal_gas.d:98-139)
__device__ __forceinline__ void back_cell(const AdjArgs& a, long long g) {
    double U[5];
    for (int q = 0; q < 5; ++q) U[q] = a.U[q * a.total + g];
    double gp[NP];
    for (int m = 0; m < NP; ++m) gp[m] = a.gP[m * a.total + g];
    const double rho = U[0], dinv = 1.0 / rho;
    const double v0 = U[1] * dinv, v1 = U[2] * dinv, v2 = U[3] * dinv;
    const double u = U[4] * dinv - 0.5 * (v0 * v0 + v1 * v1 + v2 * v2);
    const double T = u * a.P.gas.Cvinv;
    const double gR = a.P.gas.gamma * a.P.gas.R;
    const double aa = sqrt(gR * T);
    double gu = gp[4] + gp[5] * gR * a.P.gas.Cvinv / (2.0 * aa);
    double gv0 = gp[1] - gu * v0, gv1 = gp[2] - gu * v1, gv2 = gp[3] - gu * v2;
    double gdinv = gu * U[4] + gv0 * U[1] + gv1 * U[2] + gv2 * U[3];
    const double r[5] = {gp[0] - gdinv * dinv * dinv, gv0 * dinv, gv1 * dinv, gv2 * dinv, gu * dinv};
    if (a.mode == 0) {
        for (int q = 0; q < 5; ++q) a.gU[q * a.total + g] = r[q];
    } else if (a.mode == 1) {
        // predictor-corrector adjoint, first product: r = mu = J(U1)^T (dt/2 lam)
        for (int q = 0; q < 5; ++q) {
            const double l = a.lam[q * a.total + g];
            a.bbuf[q * a.total + g] = 0.5 * a.dt * l + a.dt * r[q];
            a.lam[q * a.total + g] = l + r[q];
        }
    } else {
        // second product: r = J(U0)^T b
        for (int q = 0; q < 5; ++q) a.lam[q * a.total + g] += r[q];
    }
}


__global__ void adj_decode_back_kernel(AdjArgs a) {
    long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g < a.total) back_cell(a, g);
}

// The reverse decode of one product and the decode of the next, in one pass per
// cell (the cell's cotangent gP is read, then cleared for the next product).
__global__ void adj_back_decode_kernel(AdjArgs back, AdjArgs next) {
    long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= back.total) return;
    back_cell(back, g);
    decode_cell(next, g);
}

}  // namespace

}  // namespace gdfv

using namespace gdfv;

namespace {

// The face kernel of the context's flux calculator (with the rare rules when some
// exchange rotates, some face is an outflow boundary of its own or the limiter is lmr's)
// over nb[d] CTAs of each direction.
template <int FLUX>
void launch_faces_flux(const AdjArgs& a, bool rare, const unsigned* nb, cudaStream_t s) {
    const unsigned n = nb[0] + nb[1] + nb[2];
    if (rare) adj_faces_kernel<FLUX, true><<<n, FACE_CTA, 0, s>>>(a, nb[0], nb[1]);
    else adj_faces_kernel<FLUX, false><<<n, FACE_CTA, 0, s>>>(a, nb[0], nb[1]);
}

void launch_faces(const AdjArgs& a, int flux, const unsigned* nb, cudaStream_t s) {
    const bool rare = a.P.rotating || a.P.outflow_bcs || a.P.lmr_epsilon || a.P.graded;
    if (flux == FLUX_HLLC) launch_faces_flux<FLUX_HLLC>(a, rare, nb, s);
    else launch_faces_flux<FLUX_AUSMDV>(a, rare, nb, s);
}

// The forms the VJP, step and rollout adjoints take.
bool vjp_supported(int ctx, const AdjView& v) {
    if (!v.prepared) { adjoint_set_error(ctx, "call gdfv_prepare first"); return false; }
    if (v.mhd) {
        for (const BlockDesc& B : v.h_blocks)
            for (int f = 0; f < 6; ++f)
                if (B.bc_type[f] == BC_FIXED_P || B.bc_type[f] == BC_FIXED_PT) {
                    adjoint_set_error(ctx, "the MHD residual VJP does not take outflow_fixed_p boundaries");
                    return false;
                }
        return true;
    }
    if (v.flux != FLUX_AUSMDV && v.flux != FLUX_HLLC) {
        adjoint_set_error(ctx, "the adjoint supports flux_calculator=ausmdv or hllc (and hlle with MHD in "
                               "gdfv_residual_vjp)");
        return false;
    }
    return true;
}

// Scratch layout, np = 6 primitives (Euler) or 10 (MHD), nq conserved quantities:
// P [np][total] | gP [np][total] | b [nq][total] | face offsets [3][nblocks+1] | inflow
// cotangents [ninflow][np].  Face offsets are uploaded once per allocation.
cudaError_t vjp_setup(const AdjView& v, AdjArgs& a, std::vector<long long>& off) {
    const long long total = v.total;
    const long long np = v.mhd ? NPM : NP, nq = v.mhd ? 10 : 5;
    const long long need = (2 * np + nq) * total + 3 * (v.nblocks + 1) + np * (long long)v.ninflow + 8;
    cudaError_t e = cudaSuccess;
    if (*v.scratch_n < need) {
        if (*v.scratch) cudaFree(*v.scratch);
        *v.scratch = nullptr;
        *v.scratch_n = 0;
        *v.scratch_ready = 0;
        e = cudaMalloc((void**)v.scratch, sizeof(double) * need);
        if (e != cudaSuccess) return e;
        *v.scratch_n = need;
    }
    double* base = *v.scratch;
    a = AdjArgs{};
    a.blocks = v.d_blocks;
    a.inflow = v.d_inflow;
    a.rot = v.d_rot;
    a.Pp = base;
    a.gP = base + np * total;
    a.bbuf = base + 2 * np * total;
    a.face_off = reinterpret_cast<const long long*>(base + (2 * np + nq) * total);
    a.gInflow = base + (2 * np + nq) * total + 3 * (v.nblocks + 1);
    a.chd_slot = a.gInflow + np * v.ninflow;   // two doubles of the tail
    a.c_h = v.c_h;
    a.total = total;
    a.nblocks = v.nblocks;
    a.P = v.P;
    a.w_scale = 1.0;
    off.assign(3 * (v.nblocks + 1), 0);
    for (int d = 0; d < 3; ++d) {
        for (int b = 0; b < v.nblocks; ++b) {
            const BlockDesc& B = v.h_blocks[b];
            // 2D blocks have no k faces (the residual sums four faces)
            long long nf = (v.dims == 2 && d == 2) ? 0
                                                   : (long long)(B.n[0] + (d == 0)) * (B.n[1] + (d == 1)) * (B.n[2] + (d == 2));
            off[d * (v.nblocks + 1) + b + 1] = off[d * (v.nblocks + 1) + b] + nf;
        }
    }
    if (!*v.scratch_ready) {
        e = cudaMemcpy((void*)a.face_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        *v.scratch_ready = 1;
    }
    return cudaSuccess;
}

// The MHD residual VJP: decode, the face sweep of the three directions, reverse decode.
cudaError_t enqueue_vjp_mhd(const AdjView& v, const AdjArgs& a, const std::vector<long long>& off) {
    const int nt = 256;
    const unsigned nb_cells = (unsigned)((v.total + nt - 1) / nt);
    adj_decode_mhd_kernel<<<nb_cells, nt, 0, v.stream>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    unsigned nb[3];
    for (int d = 0; d < 3; ++d) nb[d] = (unsigned)((off[d * (v.nblocks + 1) + v.nblocks] + 127) / 128);
    launch_faces_mhd(a, nb, v.stream);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    adj_back_mhd_kernel<<<nb_cells, nt, 0, v.stream>>>(a);
    return cudaGetLastError();
}

// decode, the three face sweeps (cotangents scattered onto gP) and the reverse decode.
cudaError_t enqueue_vjp(const AdjView& v, const AdjArgs& a, const std::vector<long long>& off) {
    const int nt = 256;
    const long long total = v.total;
    adj_decode_kernel<<<(unsigned)((total + nt - 1) / nt), nt, 0, v.stream>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        unsigned nb[3];
        for (int d = 0; d < 3; ++d) nb[d] = (unsigned)((off[d * (v.nblocks + 1) + v.nblocks] + 127) / 128);
        launch_faces(a, v.flux, nb, v.stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        adj_decode_back_kernel<<<(unsigned)((total + nt - 1) / nt), nt, 0, v.stream>>>(a);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace

extern "C" int gdfv_residual_vjp(int ctx, const double* U_dev, const double* W_dev, double* G_dev,
                                 double* g_inflow_host) {
    AdjView v;
    if (!adjoint_view(ctx, &v)) return GDFV_ERR_ARG;
    if (!vjp_supported(ctx, v)) return v.prepared ? GDFV_ERR_ARG : GDFV_ERR_STATE;
    if (!U_dev || !W_dev || !G_dev) { adjoint_set_error(ctx, "null pointer"); return GDFV_ERR_ARG; }
    AdjArgs a;
    std::vector<long long> off;
    cudaError_t e = vjp_setup(v, a, off);
    a.U = U_dev;
    a.W = W_dev;
    a.gU = G_dev;
    a.mode = 0;
    const int np = v.mhd ? NPM : NP;
    if (e == cudaSuccess && v.ninflow > 0) e = cudaMemsetAsync(a.gInflow, 0, sizeof(double) * np * v.ninflow, v.stream);
    if (e == cudaSuccess) e = v.mhd ? enqueue_vjp_mhd(v, a, off) : enqueue_vjp(v, a, off);
    if (e == cudaSuccess && g_inflow_host && v.ninflow > 0)
        e = cudaMemcpyAsync(g_inflow_host, a.gInflow, sizeof(double) * np * v.ninflow, cudaMemcpyDeviceToHost, v.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) { adjoint_set_error(ctx, cudaGetErrorString(e)); return GDFV_ERR_CUDA; }
    return GDFV_OK;
}

namespace {

// A chain of products: the reverse decode of each product runs fused with the
// decode of the next one (adj_back_decode_kernel, or its MHD form); finish() ends
// the chain.
struct VjpChain {
    bool pending = false;
    AdjArgs back{};
    cudaError_t product(const AdjView& v, const AdjArgs& a, const std::vector<long long>& off) {
        const int nt = 256;
        const unsigned nb_cells = (unsigned)((v.total + nt - 1) / nt);
        if (v.mhd) {
            if (pending) adj_back_decode_mhd_kernel<<<nb_cells, nt, 0, v.stream>>>(back, a);
            else adj_decode_mhd_kernel<<<nb_cells, nt, 0, v.stream>>>(a);
        } else {
            if (pending) adj_back_decode_kernel<<<nb_cells, nt, 0, v.stream>>>(back, a);
            else adj_decode_kernel<<<nb_cells, nt, 0, v.stream>>>(a);
        }
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
            unsigned nb[3];
            for (int d = 0; d < 3; ++d) nb[d] = (unsigned)((off[d * (v.nblocks + 1) + v.nblocks] + 127) / 128);
            if (v.mhd) launch_faces_mhd(a, nb, v.stream);
            else launch_faces(a, v.flux, nb, v.stream);
            e = cudaGetLastError();
        }
        back = a;
        pending = true;
        return e;
    }
    cudaError_t finish(const AdjView& v) {
        if (!pending) return cudaSuccess;
        pending = false;
        const int nt = 256;
        const unsigned nb_cells = (unsigned)((v.total + nt - 1) / nt);
        if (v.mhd) adj_back_mhd_kernel<<<nb_cells, nt, 0, v.stream>>>(back);
        else adj_decode_back_kernel<<<nb_cells, nt, 0, v.stream>>>(back);
        return cudaGetLastError();
    }
};

// The adjoint of one predictor-corrector step, enqueued on v.stream:
// mu = J(U1)^T (dt/2 lam); b = dt/2 lam + dt mu; lam += mu; then lam += J(U0)^T b.
// MHD with cleaning: the step's c_h and psi damping factor are formed first from U0
// (as gdfv_run forms them at the step's start); the corrector evaluated R at U1 with
// psi damped, and damped psi again in U2:
//   U2 = D (U0 + dt/2 R(U0) + dt/2 R(D U1)),  U1 = U0 + dt R(U0),
// so lam' = D lam, mu = J(D U1)^T (dt/2 lam'), b = dt/2 lam' + dt D mu,
// lam <- lam' + D mu + J(U0)^T b (the mode-1 decode and reverse decode apply D).
cudaError_t enqueue_step_adjoint(int ctx, const AdjView& v, AdjArgs a, const std::vector<long long>& off,
                                 const double* U0, const double* U1, double dt, double* lam, VjpChain& chain) {
    a.chd = nullptr;
    if (v.mhd && v.P.divergence_cleaning) {
        cudaError_t e = enqueue_step_ch(ctx, v.stream, U0, dt, a.chd_slot);
        if (e != cudaSuccess) return e;
        a.chd = a.chd_slot;
    }
    a.lam = lam;
    a.dt = dt;
    a.U = U1;
    a.W = lam;
    a.w_scale = 0.5 * dt;
    a.mode = 1;
    cudaError_t e = chain.product(v, a, off);
    a.U = U0;
    a.W = a.bbuf;
    a.w_scale = 1.0;
    a.mode = 2;
    if (e == cudaSuccess) e = chain.product(v, a, off);
    return e;
}

}  // namespace

extern "C" int gdfv_step_adjoint(int ctx, const double* U0_dev, const double* U1_dev, double dt, double* lam_dev,
                                 double* g_inflow_dev) {
    AdjView v;
    if (!adjoint_view(ctx, &v)) return GDFV_ERR_ARG;
    if (!vjp_supported(ctx, v)) return v.prepared ? GDFV_ERR_ARG : GDFV_ERR_STATE;
    if (!U0_dev || !U1_dev || !lam_dev || (v.ninflow > 0 && !g_inflow_dev) || !(dt > 0.0)) {
        adjoint_set_error(ctx, "gdfv_step_adjoint needs U0, U1, lam (and g_inflow with inflow faces) and dt > 0");
        return GDFV_ERR_ARG;
    }
    if (v.mhd && v.P.divergence_cleaning) {   // the scan scratch of the step's c_h
        const int st = steps_dt_prepare(ctx);
        if (st) return st;
    }
    AdjArgs a;
    std::vector<long long> off;
    cudaError_t e = vjp_setup(v, a, off);
    if (v.ninflow > 0) a.gInflow = g_inflow_dev;
    VjpChain chain;
    if (e == cudaSuccess) e = enqueue_step_adjoint(ctx, v, a, off, U0_dev, U1_dev, dt, lam_dev, chain);
    if (e == cudaSuccess) e = chain.finish(v);
    if (e != cudaSuccess) { adjoint_set_error(ctx, cudaGetErrorString(e)); return GDFV_ERR_CUDA; }
    return GDFV_OK;
}

extern "C" int gdfv_rollout_adjoint(int ctx, const double* const* ckpt_dev, int n_ckpt, const double* dts, int nsteps,
                                    int checkpoint_every, double* const* work_dev, int last_ready, double* lam_dev,
                                    double* g_inflow_dev) {
    AdjView v;
    if (!adjoint_view(ctx, &v)) return GDFV_ERR_ARG;
    if (!vjp_supported(ctx, v)) return v.prepared ? GDFV_ERR_ARG : GDFV_ERR_STATE;
    const int K = checkpoint_every;
    if (!ckpt_dev || !dts || !work_dev || !lam_dev || (v.ninflow > 0 && !g_inflow_dev) || nsteps < 1 || K < 1 ||
        K > 64 || n_ckpt != (nsteps + K - 1) / K) {
        adjoint_set_error(ctx, "gdfv_rollout_adjoint: needs one checkpoint per segment of checkpoint_every (<= 64) "
                               "steps, 4*checkpoint_every work arrays, lam (and g_inflow with inflow faces)");
        return GDFV_ERR_ARG;
    }
    for (int m = 0; m < 4 * K; ++m)
        if (!work_dev[m]) { adjoint_set_error(ctx, "gdfv_rollout_adjoint: null work array"); return GDFV_ERR_ARG; }
    for (int m = 0; m < nsteps; ++m)
        if (!(dts[m] > 0.0)) { adjoint_set_error(ctx, "gdfv_rollout_adjoint: dt must be > 0"); return GDFV_ERR_ARG; }
    int st = steps_dt_prepare(ctx);
    if (st) return st;
    AdjArgs a;
    std::vector<long long> off;
    cudaError_t e = vjp_setup(v, a, off);
    if (v.ninflow > 0) a.gInflow = g_inflow_dev;
    cudaStream_t aux = context_aux_stream(ctx, 0);     // recomputation, lowest priority
    AdjView vh = v;                                    // adjoint sweep, highest priority
    vh.stream = context_aux_stream(ctx, 1);
    if (e == cudaSuccess && (!aux || !vh.stream)) e = cudaErrorNotReady;
    // Work arrays: two sets of (K states, K predictor states); segment s uses set
    // (nseg-1-s) % 2.  The recomputation of segment s-1 (aux stream) runs while the
    // adjoint of segment s (context stream) runs; events order the reuse of a set.
    cudaEvent_t start = nullptr, rec_done[2] = {nullptr, nullptr}, adj_done[2] = {nullptr, nullptr};
    for (cudaEvent_t* ev : {&start, &rec_done[0], &rec_done[1], &adj_done[0], &adj_done[1]})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    const int nseg = n_ckpt;
    auto seg_len = [&](int s) { return std::min(K, nsteps - s * K); };
    bool first = true;
    auto recompute = [&](int s, int p) -> cudaError_t {
        // the state after a segment's last step is the next checkpoint: not recomputed
        double* outs[64];
        const int len = seg_len(s);
        for (int m = 0; m < len; ++m) outs[m] = m < len - 1 ? work_dev[2 * K * p + m] : nullptr;
        cudaError_t r = enqueue_steps_dt(ctx, aux, ckpt_dev[s], outs, work_dev + 2 * K * p + K,
                                         dts + (size_t)s * K, len, first);
        first = false;
        if (r == cudaSuccess) r = cudaEventRecord(rec_done[p], aux);
        return r;
    };
    if (e == cudaSuccess) e = cudaEventRecord(start, v.stream);   // inputs written on the context stream
    if (e == cudaSuccess) e = cudaStreamWaitEvent(aux, start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(vh.stream, start, 0);
    VjpChain chain;
    // the last segment's states and predictor states may come from the forward pass
    if (e == cudaSuccess) e = last_ready ? cudaEventRecord(rec_done[0], aux) : recompute(nseg - 1, 0);
    for (int idx = 0; idx < nseg && e == cudaSuccess; ++idx) {
        const int s = nseg - 1 - idx, p = idx % 2, q = 1 - p;
        if (s >= 1) {
            if (idx >= 1) e = cudaStreamWaitEvent(aux, adj_done[q], 0);   // set q free again
            if (e == cudaSuccess) e = recompute(s - 1, q);
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(vh.stream, rec_done[p], 0);
        double* const* outs = work_dev + 2 * K * p;
        double* const* preds = work_dev + 2 * K * p + K;
        for (int n = seg_len(s) - 1; n >= 0 && e == cudaSuccess; --n) {
            const double* U0 = n == 0 ? ckpt_dev[s] : outs[n - 1];
            e = enqueue_step_adjoint(ctx, vh, a, off, U0, preds[n], dts[(size_t)s * K + n], lam_dev, chain);
        }
        // each segment ends its chain, so that every reader of the set precedes adj_done
        if (e == cudaSuccess) e = chain.finish(vh);
        if (e == cudaSuccess) e = cudaEventRecord(adj_done[p], vh.stream);
    }
    if (e == cudaSuccess) {
        if (!first) st = steps_dt_status(ctx, aux);   // failure counters of the recomputed segments
        else e = cudaStreamSynchronize(aux);
        if (st == GDFV_OK && e == cudaSuccess) e = cudaStreamSynchronize(vh.stream);
    }
    for (cudaEvent_t ev : {start, rec_done[0], rec_done[1], adj_done[0], adj_done[1]})
        if (ev) cudaEventDestroy(ev);
    if (e != cudaSuccess) { adjoint_set_error(ctx, cudaGetErrorString(e)); return GDFV_ERR_CUDA; }
    return st;
}
