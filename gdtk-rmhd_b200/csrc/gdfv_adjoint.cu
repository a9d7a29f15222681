// gdfv_adjoint.cu -- hand-written vector-Jacobian product of the residual,
// g = (dR/dU)^T w, for the Euler path with the ausmdv flux (FP64).
//
// The residual (e4/fvcell.d:824-856) is R_c = (1/V) sum_faces +-A F_f, each face
// flux F_f a function of the four stencil states (e4/onedinterp.d:751-989 and
// e4/fluxcalc.d:477-651), each state a function of U through decode_conserved
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

#include <string>
#include <vector>

#include "../../include/gdfv.h"
#include "gdfv_internal.h"
#include "gdfv_launch.h"

namespace gdfv {

namespace {

constexpr int NP = 6;  // rho, v0, v1, v2, u, a

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
};

__device__ __forceinline__ void l2r2_fwd(const double* w, const NumParams& P, double q1, double q0, double r0,
                                         double r1, double& qL, double& qR, L2R2Rec& t) {
    t.dLm = (q0 - q1) * w[W_TOL];
    t.del = (r0 - q0) * w[W_TOC];
    t.dRp = (r1 - r0) * w[W_TOR];
    t.sL = 1.0; t.sR = 1.0;
    const double eps = P.eps_van_albada;
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
    }
    g0 += gdLm * w[W_TOL]; g1 -= gdLm * w[W_TOL];
    h0 += gdel * w[W_TOC]; g0 -= gdel * w[W_TOC];
    h1 += gdRp * w[W_TOR]; h0 -= gdRp * w[W_TOR];
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
    double pLplus, uLplus;
    if (subL) { pLplus = L.p * (ML + 1.0) * (ML + 1.0) * (2.0 - ML) * 0.25; uLplus = alphaL * (QL - duL) + duL; }
    else { pLplus = L.p * duL * rcp(L.u); uLplus = duL; }
    double duR = 0.5 * (R.u - fabs(R.u));
    bool subR = fabs(MR) <= 1.0;
    double QR = -(R.u - am) * (R.u - am) * (0.25 * iam);
    double pRminus, uRminus;
    if (subR) { pRminus = R.p * (MR - 1.0) * (MR - 1.0) * (2.0 + MR) * 0.25; uRminus = alphaR * (QR - duR) + duR; }
    else { pRminus = R.p * duR * rcp(R.u); uRminus = duR; }
    (void)pLplus; (void)pRminus;  // p_half enters F linearly: only its cotangent is needed
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

struct AdjArgs {
    const BlockDesc* blocks;
    const InflowState* inflow;
    const double* U;
    const double* W;
    double* Pp;        // [6][total]
    double* gP;        // [6][total]
    double* gU;        // [nq][total]
    double* gInflow;   // [ninflow][6]
    const long long* face_off;  // [3][nblocks+1] prefix counts of faces per direction
    double* lam;       // [nq][total] adjoint state of a fused step (modes 1, 2)
    double* bbuf;      // [nq][total] b = dt/2 lam + dt mu (mode 1 writes, mode 2 is its W)
    double w_scale;    // W enters scaled by this
    double dt;
    long long total;
    int nblocks;
    int mode;          // 0: gU = result; 1: mu -> bbuf, lam += mu; 2: lam += result
    NumParams P;
};

__global__ void adj_decode_kernel(AdjArgs a) {
    long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= a.total) return;
    double u[5];
    for (int q = 0; q < 5; ++q) u[q] = a.U[q * a.total + g];
    Prim<double> s;
    double p, T;
    decode(a.P, u, s, p, T);
    double v[NP] = {s.rho, s.v[0], s.v[1], s.v[2], s.u, s.a};
    for (int m = 0; m < NP; ++m) { a.Pp[m * a.total + g] = v[m]; a.gP[m * a.total + g] = 0.0; }
}

// Stencil cell state from P (with the ghost maps) and the reverse map of a cotangent.
struct Src {
    const BlockDesc* blk;
    long long c0, c1;
    int kind, axis, inflow;
};

__device__ Src adj_resolve(const AdjArgs& a, const BlockDesc& B, int i, int j, int k) {
    StageArgs A{};
    A.blocks = a.blocks;
    CellSrc s = resolve(A, B, i, j, k);
    return Src{s.blk, s.c0, s.c1, s.kind, s.axis, s.inflow};
}

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
}

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
    for (int m = 0; m < NP; ++m) {
        double v = gc[m];
        if (s.kind == SRC_MIRROR && m == 1 + s.axis) v = -v;
        atomicAdd(&a.gP[m * a.total + g0], v);
    }
}

template <int D>
__global__ void __launch_bounds__(128, 3) adj_face_kernel(AdjArgs a) {
    long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long* off = a.face_off + D * (a.nblocks + 1);
    if (f >= off[a.nblocks]) return;
    int b = 0;
    while (off[b + 1] <= f) ++b;
    const BlockDesc& B = a.blocks[b];
    long long lf = f - off[b];
    int nf0 = B.n[0] + (D == 0), nf1 = B.n[1] + (D == 1);
    int i = (int)(lf % nf0);
    int j = (int)((lf / nf0) % nf1);
    int k = (int)(lf / ((long long)nf0 * nf1));
    // stencil: cells at index-2, -1, 0, +1 along D (left cells below the face index)
    int ci[4], cj[4], ck[4];
    for (int m = 0; m < 4; ++m) {
        ci[m] = i - (D == 0 ? 2 - m : 0); cj[m] = j - (D == 1 ? 2 - m : 0); ck[m] = k - (D == 2 ? 2 - m : 0);
    }
    Src s[4];
    double c[4][NP];
    for (int m = 0; m < 4; ++m) {
        s[m] = adj_resolve(a, B, ci[m], cj[m], ck[m]);
        adj_load(a, s[m], c[m]);
    }
    // cotangent of the face flux: F enters R_right with +A/V and R_left with -A/V
    const double AV = B.area[D] * B.vol_inv * a.w_scale;
    const int nD = B.n[D];
    const int idxD = D == 0 ? i : (D == 1 ? j : k);
    const bool leftIn = idxD - 1 >= 0, rightIn = idxD < nD;
    const long long gl = B.offset + (long long)(i - (D == 0)) + (long long)B.n[0] * ((long long)(j - (D == 1)) + (long long)B.n[1] * (k - (D == 2)));
    const long long gr = B.offset + (long long)i + (long long)B.n[0] * ((long long)j + (long long)B.n[1] * k);
    double gFg[5];
    for (int q = 0; q < 5; ++q) {
        double wr = rightIn ? a.W[q * a.total + gr] : 0.0;
        double wl = leftIn ? a.W[q * a.total + gl] : 0.0;
        gFg[q] = AV * (wr - wl);
    }
    constexpr int ax0 = D, ax1 = (D + 1) % 3, ax2 = (D + 2) % 3;
    double gF[5] = {gFg[MASS], gFg[XMOM + ax0], gFg[XMOM + ax1], gFg[XMOM + ax2], gFg[TOTENERGY]};
    // ---- forward reconstruction (local-frame scalars: vn, vt1, vt2, rho, u)
    const double* w = B.w[D];
    const NumParams& P = a.P;
    const int pv[5] = {1 + ax0, 1 + ax1, 1 + ax2, 0, 4};
    double qL[5], qR[5];
    for (int sc = 0; sc < 5; ++sc) {
        L2R2Rec rec;  // recomputed in the reverse sweep rather than kept live
        l2r2_fwd(w, P, c[0][pv[sc]], c[1][pv[sc]], c[2][pv[sc]], c[3][pv[sc]], qL[sc], qR[sc], rec);
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
    ausmdv_vjp(P, L, Rs, gF, gL, gR);
    double gc[4][NP];
    for (int m = 0; m < 4; ++m)
        for (int q = 0; q < NP; ++q) gc[m][q] = 0.0;
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
        L2R2Rec rec;
        double ql, qr;
        l2r2_fwd(w, P, c[0][v], c[1][v], c[2][v], c[3][v], ql, qr, rec);
        l2r2_rev(w, P, c[0][v], c[1][v], c[2][v], c[3][v], rec, gqL[sc], gqR[sc], gc[0][v], gc[1][v], gc[2][v],
                 gc[3][v]);
    }
    for (int m = 0; m < 4; ++m) adj_scatter(a, s[m], gc[m]);
}

// gU = (dP/dU)^T gP for P = decode(U) (e4/fvcell.d:586-822 with ideal_gas.d:98-139)
__global__ void adj_decode_back_kernel(AdjArgs a) {
    long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= a.total) return;
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

}  // namespace

}  // namespace gdfv

using namespace gdfv;

namespace {

bool vjp_supported(int ctx, const AdjView& v) {
    if (!v.prepared) { adjoint_set_error(ctx, "call gdfv_prepare first"); return false; }
    if (v.mhd || v.flux != FLUX_AUSMDV || v.dims != 3) {
        adjoint_set_error(ctx, "the adjoint supports the 3D Euler path with flux_calculator=ausmdv");
        return false;
    }
    return true;
}

// Scratch layout: P [6][total] | gP [6][total] | b [5][total] | face offsets [3][nblocks+1]
// | inflow cotangents [ninflow][6].  Face offsets are uploaded once per allocation.
cudaError_t vjp_setup(const AdjView& v, AdjArgs& a, std::vector<long long>& off) {
    const long long total = v.total;
    const long long need = 17 * total + 3 * (v.nblocks + 1) + 6 * (long long)v.ninflow + 8;
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
    a.Pp = base;
    a.gP = base + 6 * total;
    a.bbuf = base + 12 * total;
    a.face_off = reinterpret_cast<const long long*>(base + 17 * total);
    a.gInflow = base + 17 * total + 3 * (v.nblocks + 1);
    a.total = total;
    a.nblocks = v.nblocks;
    a.P = v.P;
    a.w_scale = 1.0;
    off.assign(3 * (v.nblocks + 1), 0);
    for (int d = 0; d < 3; ++d) {
        for (int b = 0; b < v.nblocks; ++b) {
            const BlockDesc& B = v.h_blocks[b];
            long long nf = (long long)(B.n[0] + (d == 0)) * (B.n[1] + (d == 1)) * (B.n[2] + (d == 2));
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

// decode, the three face sweeps (cotangents scattered onto gP) and the reverse decode.
cudaError_t enqueue_vjp(const AdjView& v, const AdjArgs& a, const std::vector<long long>& off) {
    const int nt = 256;
    const long long total = v.total;
    adj_decode_kernel<<<(unsigned)((total + nt - 1) / nt), nt, 0, v.stream>>>(a);
    cudaError_t e = cudaGetLastError();
    for (int d = 0; d < 3 && e == cudaSuccess; ++d) {
        long long nf = off[d * (v.nblocks + 1) + v.nblocks];
        const unsigned nb = (unsigned)((nf + 127) / 128);  // 128-thread CTAs, 3 per SM by registers
        if (d == 0) adj_face_kernel<0><<<nb, 128, 0, v.stream>>>(a);
        if (d == 1) adj_face_kernel<1><<<nb, 128, 0, v.stream>>>(a);
        if (d == 2) adj_face_kernel<2><<<nb, 128, 0, v.stream>>>(a);
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
    if (e == cudaSuccess && v.ninflow > 0) e = cudaMemsetAsync(a.gInflow, 0, sizeof(double) * 6 * v.ninflow, v.stream);
    if (e == cudaSuccess) e = enqueue_vjp(v, a, off);
    if (e == cudaSuccess && g_inflow_host && v.ninflow > 0)
        e = cudaMemcpyAsync(g_inflow_host, a.gInflow, sizeof(double) * 6 * v.ninflow, cudaMemcpyDeviceToHost, v.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) { adjoint_set_error(ctx, cudaGetErrorString(e)); return GDFV_ERR_CUDA; }
    return GDFV_OK;
}

extern "C" int gdfv_step_adjoint(int ctx, const double* U0_dev, const double* U1_dev, double dt, double* lam_dev,
                                 double* g_inflow_dev) {
    AdjView v;
    if (!adjoint_view(ctx, &v)) return GDFV_ERR_ARG;
    if (!vjp_supported(ctx, v)) return v.prepared ? GDFV_ERR_ARG : GDFV_ERR_STATE;
    if (!U0_dev || !U1_dev || !lam_dev || (v.ninflow > 0 && !g_inflow_dev) || !(dt > 0.0)) {
        adjoint_set_error(ctx, "gdfv_step_adjoint needs U0, U1, lam (and g_inflow with inflow faces) and dt > 0");
        return GDFV_ERR_ARG;
    }
    AdjArgs a;
    std::vector<long long> off;
    cudaError_t e = vjp_setup(v, a, off);
    if (v.ninflow > 0) a.gInflow = g_inflow_dev;
    a.lam = lam_dev;
    a.dt = dt;
    // mu = J(U1)^T (dt/2 lam); b = dt/2 lam + dt mu; lam += mu
    a.U = U1_dev;
    a.W = lam_dev;
    a.w_scale = 0.5 * dt;
    a.mode = 1;
    if (e == cudaSuccess) e = enqueue_vjp(v, a, off);
    // lam += J(U0)^T b
    a.U = U0_dev;
    a.W = a.bbuf;
    a.w_scale = 1.0;
    a.mode = 2;
    if (e == cudaSuccess) e = enqueue_vjp(v, a, off);
    if (e != cudaSuccess) { adjoint_set_error(ctx, cudaGetErrorString(e)); return GDFV_ERR_CUDA; }
    return GDFV_OK;
}
