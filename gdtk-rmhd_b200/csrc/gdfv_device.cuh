// gdfv_device.cuh -- device-side data structures and the per-face / per-cell
// numerics of the structured-grid finite-volume update.
//
// The arithmetic follows the reference's Eilmer-4 path (cited per function);
// the data layout is this library's own: conserved quantities in SoA FP64
// arrays (variable-major, i fastest), no ghost storage (ghost cells are
// synthesised by the tile loader from the boundary-condition table).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gdfv {

// ---------------------------------------------------------------- indices
// Conserved-quantity slots, e4/conservedquantities.d:148-197 (3D or MHD ordering)
enum : int { MASS = 0, XMOM = 1, YMOM = 2, ZMOM = 3, TOTENERGY = 4, XB = 5, YB = 6, ZB = 7, PSI = 8, DIVB = 9 };
enum : int { FLUX_AUSMDV = 0, FLUX_HLLC = 1, FLUX_HLLE = 2 };
enum : int { BC_SLIP_WALL = 0, BC_EXTRAPOLATE = 1, BC_INFLOW = 2, BC_EXCHANGE = 3, BC_FIXED_P = 4, BC_FIXED_PT = 5,
             BC_SIMPLE_FLUX = 6 };
// step status words
enum : int { ST_OK = 0, ST_DECODE_FAILED = 1, ST_TOO_MANY_BAD_CELLS = 2 };

// weights of the l2r2 reconstruction for one index direction (e4/onedinterp.d:338-355),
// precomputed on the host because every cell of a block has the same lengths
enum : int { W_AL0 = 0, W_AR0, W_LENL0, W_LENR0, W_TOL, W_TOC, W_TOR, W_TWOL, W_TWOR, W_N };
// per-cell weights of a graded block along one index direction: the two interface values
// of cell c (face c+1/2 left state, face c-1/2 right state) come from l2r2_prepare's
// weights of those two faces, which are these expressions of len(c-1), len(c), len(c+1)
enum : int { GW_TOL = 0,  // 2/(len_c + len_{c-1})
             GW_TOC,      // 2/(len_{c+1} + len_c)
             GW_A,        // 0.5 len_c / (len_{c-1} + 2 len_c + len_{c+1})  (aL0 of face c+1/2, aR0 of c-1/2)
             GW_TWOL,     // 2 len_c + len_{c-1}
             GW_LENR0,    // len_{c+1}
             GW_LENL0,    // len_{c-1}
             GW_TWOR,     // 2 len_c + len_{c+1}
             GW_N };

struct GasParams {
    double R, gamma, Cv, Cvinv;
};

struct NumParams {
    GasParams gas;
    double eps_van_albada;
    double divB_damping_length;
    double max_velocity, max_temp, min_temp;
    int apply_limiter, extrema_clipping, apply_entropy_fix, glm_reference_indexing;
    int mhd, divergence_cleaning, dims, stringent_cfl;
    int nq;
    int lmr_epsilon;    // van Albada epsilon scaled per face (lmr/onedinterp.d:147-151)
    int outflow_bcs;    // some face has OutFlowBC_FixedP, _FixedPT or _SimpleFlux
    int graded;         // some block has cell lengths varying along an axis
    int rotating;       // some exchange face rotates its ghosts' vectors (Rmatrix)
};

// Fixed ghost state of a supersonic-inflow face (FlowStateCopy, flow_state_copy.d:92-107)
struct InflowState {
    double rho, vel[3], u, p, a, B[3], psi;
};

struct BlockDesc {
    int n[3];             // nic, njc, nkc
    int pad0_;
    long long offset;     // first cell of this block in the SoA arrays
    double len[3];        // dx, dy, dz
    double area[3];       // face areas normal to i, j, k
    double vol_inv;
    double L_min;
    double x0, y0, z0;
    double w[3][W_N];     // l2r2 weights per direction
    int bc_type[6], bc_xorder[6], bc_other[6], bc_other_face[6], bc_inflow[6];
    // exchange faces: the partner's cell (index within its block) that feeds the ghost
    // (i, j, k) is x[0] + x[1] i + x[2] j + x[3] k (every partner index is this block's
    // i, j, k or the ghost's depth, possibly counted from the far end: affine in i, j, k);
    // bc_xrot = 1 + the index of the rotation of the ghost's vectors in StageArgs::rot,
    // 0 for none
    int bc_xlin[6][4];
    int bc_xrot[6];
    int graded;           // rectilinear block with cell lengths varying along each axis
    // graded: cell lengths of cells -2 .. n+1 (index c + 2), ghosts as the boundary gives
    // them, and the l2r2 weights of cells -1 .. n (index (c + 1) * GW_N), per direction
    const double* glen[3];
    const double* gw[3];
};

struct TileDesc {
    int block, i0, j0, k0, k1, pad_[3];
};

// Device-resident control record: the whole step (dt rule included) runs
// without host round trips, so a batch of steps can be replayed as a graph.
struct Control {
    double time, dt_global, c_h, cfl_max, dt_allow;
    double max_time;     // stop once time >= max_time (<= 0: no limit)
    double t0;           // time at the start of the step being attempted
    double pad0_;
    long long first_bad_cell;  // global index of a cell that failed to decode
    int step, step_limit, status, halted;
    int n_fail;                // decode failures in the current attempt (retry)
    int n_invalid1, n_invalid2;  // check_data failures after stage 1 / stage 2 (abort)
    int attempt, retrying, steps_done;
    unsigned int tile_next, tile_done;  // work queue of a persistent stage launch (0 between launches)
};

// ---------------------------------------------------------------- state structs
// Cell-centre flow state as used by reconstruction (global frame).
template <class R>
struct Prim {
    R rho, v[3], u, a;
    R B[3], psi;
};

// ---------------------------------------------------------------- small helpers
// Cell lengths of cell (i, j, k) of a block (the same for every cell of a uniform block).
__device__ __forceinline__ void cell_lengths(const BlockDesc& B, int i, int j, int k, double* L) {
    if (B.graded) {
        L[0] = B.glen[0][i + 2];
        L[1] = B.glen[1][j + 2];
        L[2] = B.glen[2][k + 2];
    } else {
        L[0] = B.len[0]; L[1] = B.len[1]; L[2] = B.len[2];
    }
}

__device__ __forceinline__ double d_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double d_mul(double a, double b) { return __dmul_rn(a, b); }

template <class R> __device__ __forceinline__ R rabs(R x) { return fabs(x); }
template <> __device__ __forceinline__ float rabs<float>(float x) { return fabsf(x); }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return fmin(a, b); }
template <> __device__ __forceinline__ float rmin<float>(float a, float b) { return fminf(a, b); }
template <class R> __device__ __forceinline__ R rmax(R a, R b) { return fmax(a, b); }
template <> __device__ __forceinline__ float rmax<float>(float a, float b) { return fmaxf(a, b); }
template <class R> __device__ __forceinline__ R rsqrt_(R x) { return sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return sqrtf(x); }

// Dipole field that an MHD slip-wall ghost at (x, y) with |x| < 0.4136 takes
// (e4/bc/ghost_cell_effect/internal_copy_then_reflect.d:140-143).  The reference
// writes D's `^^`; with an integer exponent that is std.math.pow(F, int), which
// multiplies by repeated squaring: s^^2 = s*s, s^^3 = s*(s*s), s^^5 = s*((s*s)*(s*s)).
// ^^0.5 is the square root.  Written as those products here and in the oracle, in
// FP64 without contraction, both sides give the same bits.
__device__ __forceinline__ void dipole_field(double x, double y, double& Bx, double& By) {
    const double xs = x + 0., ys = y + 0.0;
    const double x2 = d_mul(xs, xs), y2 = d_mul(ys, ys);
    const double r = sqrt(d_add(x2, y2));
    const double r2 = d_mul(r, r);
    const double r5 = d_mul(r, d_mul(r2, r2));
    const double h = 0.82 / 2;
    const double h3 = d_mul(h, d_mul(h, h));
    const double cc = d_mul(0.1, h3) / d_mul(2.0, r5);
    Bx = -cc * __dsub_rn(d_mul(2.0, x2), y2);
    By = -cc * d_mul(d_mul(3.0, xs), ys);
}

// src/nm/limiters.d:41-50
template <class R>
__device__ __forceinline__ R clip_to_limits(R q, R A, R B) {
    R lower = (A <= B) ? A : B;
    R upper = (A > B) ? A : B;
    R qc = (q > lower) ? q : lower;
    return (qc <= upper) ? qc : upper;
}

// e4/onedinterp.d:357-386 interp_l2r2_scalar (beta = 1)
template <class R>
__device__ __forceinline__ void l2r2(const R* w, const NumParams& P, R qL1, R qL0, R qR0, R qR1, R& qL, R& qR) {
    R delLminus = (qL0 - qL1) * w[W_TOL];
    R del = (qR0 - qL0) * w[W_TOC];
    R delRplus = (qR1 - qR0) * w[W_TOR];
    R sL = R(1.0), sR = R(1.0);
    if (P.apply_limiter) {
        const R eps = R(P.eps_van_albada);
        sL = (delLminus * del + rabs(delLminus * del) + eps) / (delLminus * delLminus + del * del + eps);
        sR = (del * delRplus + rabs(del * delRplus) + eps) / (del * del + delRplus * delRplus + eps);
    }
    qL = qL0 + sL * w[W_AL0] * (del * w[W_TWOL] + delLminus * w[W_LENR0]);
    qR = qR0 - sR * w[W_AR0] * (delRplus * w[W_LENL0] + del * w[W_TWOR]);
    if (P.extrema_clipping) {
        qL = clip_to_limits(qL, qL0, qR0);
        qR = clip_to_limits(qR, qL0, qR0);
    }
}

// Interface state in the face-local frame: vel[0], B[0] normal.
template <class R>
struct FaceState {
    R rho, p, u, a, v[3], B[3], psi;
};

// e4/fluxcalc.d:477-651 ausmdv (factor = 1)
template <class R>
__device__ __forceinline__ void ausmdv(const NumParams& P, const FaceState<R>& L, const FaceState<R>& Rt, R* F) {
    R rL = L.rho, pL = L.p, pLrL = pL / rL;
    R uL = L.v[0], vL = L.v[1], wL = L.v[2];
    R eL = L.u, aL = L.a;
    R keL = R(0.5) * (uL * uL + vL * vL + wL * wL);
    R HL = eL + pLrL + keL;
    R rR = Rt.rho, pR = Rt.p, pRrR = pR / rR;
    R uR = Rt.v[0], vR = Rt.v[1], wR = Rt.v[2];
    R eR = Rt.u, aR = Rt.a;
    R keR = R(0.5) * (uR * uR + vR * vR + wR * wR);
    R HR = eR + pRrR + keR;
    R alphaL = R(2.0) * pLrL / (pLrL + pRrR);
    R alphaR = R(2.0) * pRrR / (pLrL + pRrR);
    R am = rmax(aL, aR);
    R ML = uL / am;
    R MR = uR / am;
    R pLplus, uLplus;
    R duL = R(0.5) * (uL + rabs(uL));
    if (rabs(ML) <= R(1.0)) {
        pLplus = pL * (ML + R(1.0)) * (ML + R(1.0)) * (R(2.0) - ML) * R(0.25);
        uLplus = alphaL * ((uL + am) * (uL + am) / (R(4.0) * am) - duL) + duL;
    } else {
        pLplus = pL * duL / uL;
        uLplus = duL;
    }
    R pRminus, uRminus;
    R duR = R(0.5) * (uR - rabs(uR));
    if (rabs(MR) <= R(1.0)) {
        pRminus = pR * (MR - R(1.0)) * (MR - R(1.0)) * (R(2.0) + MR) * R(0.25);
        uRminus = alphaR * (-(uR - am) * (uR - am) / (R(4.0) * am) - duR) + duR;
    } else {
        pRminus = pR * duR / uR;
        uRminus = duR;
    }
    R ru_half = uLplus * rL + uRminus * rR;
    R p_half = pLplus + pRminus;
    R dp = pL - pR;
    dp = R(10.0) * rabs(dp) / rmin(pL, pR);
    R s = R(0.5) * rmin(R(1.0), dp);
    R ru2_AUSMV = uLplus * rL * uL + uRminus * rR * uR;
    R ru2_AUSMD = R(0.5) * (ru_half * (uL + uR) - rabs(ru_half) * (uR - uL));
    R ru2_half = (R(0.5) + s) * ru2_AUSMV + (R(0.5) - s) * ru2_AUSMD;
    F[MASS] = ru_half;
    F[XMOM] = ru2_half + p_half;
    if (ru_half >= R(0.0)) {
        F[YMOM] = ru_half * vL;
        F[ZMOM] = ru_half * wL;
        F[TOTENERGY] = ru_half * HL;
    } else {
        F[YMOM] = ru_half * vR;
        F[ZMOM] = ru_half * wR;
        F[TOTENERGY] = ru_half * HR;
    }
    if (P.apply_entropy_fix) {
        const R C_EFIX = R(0.125);
        bool caseA = ((uL - aL) < R(0.0)) && ((uR - aR) > R(0.0));
        bool caseB = ((uL + aL) < R(0.0)) && ((uR + aR) > R(0.0));
        R d_ua = R(0.0);
        if (caseA && !caseB) d_ua = C_EFIX * ((uR - aR) - (uL - aL));
        if (caseB && !caseA) d_ua = C_EFIX * ((uR + aR) - (uL + aL));
        if (d_ua != R(0.0)) {
            F[MASS] -= d_ua * (rR - rL);
            F[XMOM] -= d_ua * (rR * uR - rL * uL);
            F[YMOM] -= d_ua * (rR * vR - rL * vL);
            F[ZMOM] -= d_ua * (rR * wR - rL * wL);
            F[TOTENERGY] -= d_ua * (rR * HR - rL * HL);
        }
    }
}

// e4/fluxcalc.d:653-820 hllc (factor = 1, single gamma)
template <class R>
__device__ __forceinline__ void hllc(const NumParams& P, const FaceState<R>& L, const FaceState<R>& Rt, R* F) {
    const R g = R(P.gas.gamma);
    R rL = L.rho, pL = L.p, uL = L.v[0], vL = L.v[1], wL = L.v[2], eL = L.u, aL = L.a;
    R keL = R(0.5) * (uL * uL + vL * vL + wL * wL);
    R EL = rL * eL + rL * keL;
    R rR = Rt.rho, pR = Rt.p, uR = Rt.v[0], vR = Rt.v[1], wR = Rt.v[2], eR = Rt.u, aR = Rt.a;
    R keR = R(0.5) * (uR * uR + vR * vR + wR * wR);
    R ER = rR * eR + rR * keR;
    R srL = rsqrt_(rL), srR = rsqrt_(rR);
    R uhat = (srL * uL + srR * uR) / (srL + srR);
    R ghat = (srL * g + srR * g) / (srL + srR);
    R ahat2 = ((srL * aL * aL + srR * aR * aR) / (srL + srR)) +
              R(0.5) * (ghat - R(1.0)) * ((srL + srR) / rsqrt_((srL + srR))) * (uR - uL) * (uR - uL);
    R ahat = rsqrt_(ahat2);
    R SL = rmin(uL - aL, uhat - ahat);
    R SR = rmax(uR + aR, uhat + ahat);
    R S_star = (pR - pL + rL * uL * (SL - uL) - rR * uR * (SR - uR)) / (rL * (SL - uL) - rR * (SR - uR));
    bool star;
    R coeff, r, p, u, v, w, E, S;
    if (S_star > R(0.0)) {
        r = rL; p = pL; u = uL; v = vL; w = wL; E = EL; S = SL;
        if (SL > R(0.0)) { star = false; coeff = R(0.0); }
        else { star = true; coeff = rL * (SL - uL) / (SL - S_star); }
    } else {
        r = rR; p = pR; u = uR; v = vR; w = wR; E = ER; S = SR;
        if (SR < R(0.0)) { star = false; coeff = R(0.0); }
        else { star = true; coeff = rR * (SR - uR) / (SR - S_star); }
    }
    R F_mass = r * u;
    F[MASS] = star ? F_mass + S * (coeff - r) : F_mass;
    R F_momx = r * u * u + p, F_momy = r * u * v, F_momz = r * u * w;
    if (star) {
        F[XMOM] = F_momx + S * (coeff * S_star - r * u);
        F[YMOM] = F_momy + S * (coeff * v - r * v);
        F[ZMOM] = F_momz + S * (coeff * w - r * w);
    } else {
        F[XMOM] = F_momx; F[YMOM] = F_momy; F[ZMOM] = F_momz;
    }
    R F_totenergy = u * (E + p);
    if (star) {
        R U_star_totenergy = coeff * (E / r + (S_star - u) * (S_star + p / (r * (S - u))));
        F[TOTENERGY] = F_totenergy + S * (U_star_totenergy - E);
    } else {
        F[TOTENERGY] = F_totenergy;
    }
}

// e4/fluxcalc.d:1608-1780 hlle for ideal MHD (mu0 = 1)
template <class R>
__device__ __forceinline__ void hlle_mhd(const NumParams& P, const FaceState<R>& L, const FaceState<R>& Rt, R* F) {
    auto SAFESQRT = [](R x) -> R { return (rabs(x) > R(1.0e-14)) ? rsqrt_(x) : R(0.0); };
    R rL = L.rho, pL = L.p, uL = L.v[0], vL = L.v[1], wL = L.v[2];
    R BxL = L.B[0], ByL = L.B[1], BzL = L.B[2];
    R rR = Rt.rho, pR = Rt.p, uR = Rt.v[0], vR = Rt.v[1], wR = Rt.v[2];
    R BxR = Rt.B[0], ByR = Rt.B[1], BzR = Rt.B[2];
    const R Cv = R(P.gas.Cv), Rg = R(P.gas.R);
    R rLsqrt = rsqrt_(rL), rRsqrt = rsqrt_(rR);
    R alpha = rLsqrt / (rLsqrt + rRsqrt);
    R cv = alpha * Cv + (R(1.0) - alpha) * Cv;
    R Rgas = alpha * Rg + (R(1.0) - alpha) * Rg;
    R cp = cv + Rgas;
    R gam = cp / cv;
    R rho = R(0.5) * (rL + rR);
    R p = R(0.5) * (pL + pR);
    R u = R(0.5) * (uL + uR);
    R Bx = R(0.5) * (BxL + BxR), By = R(0.5) * (ByL + ByR), Bz = R(0.5) * (BzL + BzR);
    R a2 = gam * p / rho;
    R Bx2 = Bx * Bx;
    R Bt2 = By * By + Bz * Bz;
    R BB = Bx2 + Bt2;
    R ca2 = Bx2 / rho;
    R alf = a2 + BB / rho;
    R als = SAFESQRT(alf * alf - R(4.0) * a2 * ca2);
    R cf2 = R(0.5) * (alf + als);
    R cf = rsqrt_(cf2);
    R wp = u + cf, wm = u - cf;
    R BxL2 = BxL * BxL, BtL2 = ByL * ByL + BzL * BzL, BBL = BxL2 + BtL2;
    R ptL = pL + R(0.5) * BBL;
    R uL2 = uL * uL, uuL = uL2 + vL * vL + wL * wL;
    R aL2 = gam * pL / rL, caL2 = BxL2 / rL, alfL = aL2 + BBL / rL;
    R alsL = SAFESQRT(alfL * alfL - R(4.0) * aL2 * caL2);
    R cfL2 = R(0.5) * (alfL + alsL), cfL = rsqrt_(cfL2);
    R wmL = uL - cfL;
    R BxR2 = BxR * BxR, BtR2 = ByR * ByR + BzR * BzR, BBR = BxR2 + BtR2;
    R ptR = pR + R(0.5) * BBR;
    R uR2 = uR * uR, uuR = uR2 + vR * vR + wR * wR;
    R aR2 = gam * pR / rR, caR2 = BxR2 / rR, alfR = aR2 + BBR / rR;
    R alsR = SAFESQRT(alfR * alfR - R(4.0) * aR2 * caR2);
    R cfR2 = R(0.5) * (alfR + alsR), cfR = rsqrt_(cfR2);
    R wpR = uR + cfR;
    R dU0 = rR - rL, dU1 = rR * uR - rL * uL, dU2 = rR * vR - rL * vL, dU3 = rR * wR - rL * wL;
    R dU4 = BxR - BxL, dU5 = ByR - ByL, dU6 = BzR - BzL;
    R dU7 = (pR - pL) / (gam - R(1.0)) + R(0.5) * (rR * uuR + BBR) - R(0.5) * (rL * uuL + BBL);
    R bl = rmin(wmL, wm), br = rmax(wpR, wp);
    R blm = rmin(bl, R(0.0)), brp = rmax(br, R(0.0));
    R fmassL = rL * uL, fmassR = rR * uR;
    R fmomxL = rL * uL2 - BxL2 + ptL, fmomxR = rR * uR2 - BxR2 + ptR;
    R fmomyL = rL * uL * vL - BxL * ByL, fmomyR = rR * uR * vR - BxR * ByR;
    R fmomzL = rL * uL * wL - BxL * BzL, fmomzR = rR * uR * wR - BxR * BzR;
    R fBxL = R(0.0), fBxR = R(0.0);
    R fByL = uL * ByL - vL * BxL, fByR = uR * ByR - vR * BxR;
    R fBzL = uL * BzL - wL * BxL, fBzR = uR * BzR - wR * BxR;
    R fenergyL = (rL * L.u + R(0.5) * (rL * uuL + BBL) + ptL) * uL - (uL * BxL + vL * ByL + wL * BzL) * BxL;
    R fenergyR = (rR * Rt.u + R(0.5) * (rR * uuR + BBR) + ptR) * uR - (uR * BxR + vR * ByR + wR * BzR) * BxR;
    R iden = R(1.0) / (brp - blm);
    R fac1 = brp * blm;
    F[MASS] = (brp * fmassL - blm * fmassR + fac1 * dU0) * iden;
    F[XMOM] = (brp * fmomxL - blm * fmomxR + fac1 * dU1) * iden;
    F[YMOM] = (brp * fmomyL - blm * fmomyR + fac1 * dU2) * iden;
    F[ZMOM] = (brp * fmomzL - blm * fmomzR + fac1 * dU3) * iden;
    F[TOTENERGY] = (brp * fenergyL - blm * fenergyR + fac1 * dU7) * iden;
    F[XB] = (brp * fBxL - blm * fBxR + fac1 * dU4) * iden;
    F[YB] = (brp * fByL - blm * fByR + fac1 * dU5) * iden;
    F[ZB] = (brp * fBzL - blm * fBzR + fac1 * dU6) * iden;
}

// e4/fvcell.d:586-822 decode_conserved for a single-species ideal gas.
// Returns 0 on success; nonzero where the reference throws (bad density or
// failed thermo update).  Sets p and T for the validity checks.
__device__ __forceinline__ int decode(const NumParams& P, const double* U, Prim<double>& s, double& p, double& T) {
    double rho = U[MASS];
    if (!(rho > 0.0)) return 1;
    s.rho = rho;
    double dinv = 1.0 / rho;
    s.v[0] = U[XMOM] * dinv;
    s.v[1] = U[YMOM] * dinv;
    s.v[2] = U[ZMOM] * dinv;
    double rE = U[TOTENERGY];
    if (P.mhd) {
        s.B[0] = U[XB]; s.B[1] = U[YB]; s.B[2] = U[ZB]; s.psi = U[PSI];
        double me = 0.5 * (s.B[0] * s.B[0] + s.B[1] * s.B[1] + s.B[2] * s.B[2]);
        rE = rE - me;
    } else {
        s.B[0] = s.B[1] = s.B[2] = 0.0; s.psi = 0.0;
    }
    double u = rE * dinv;
    double ke = 0.5 * (s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]);
    u = u - ke;
    s.u = u;
    // ideal_gas.d:98-106 update_thermo_from_rhou
    if (u <= 0.0 || rho <= 0.0) return 2;
    T = u * P.gas.Cvinv;
    p = rho * P.gas.R * T;
    if (T <= 0.0) return 2;
    s.a = sqrt(P.gas.gamma * P.gas.R * T);  // ideal_gas.d:132-139
    return 0;
}

// e4/flowstate.d:363-390 check_data (gas_state.d:226-266)
__device__ __forceinline__ bool check_data(const NumParams& P, const Prim<double>& s, double p, double T) {
    bool ok = true;
    if (!isfinite(s.rho) || s.rho < 1.01 * 0.0) ok = false;
    if (!isfinite(T) || T < 1.01 * 0.0) ok = false;
    if (!isfinite(p)) ok = false;
    if (!isfinite(s.a)) ok = false;
    if (fabs(s.v[0]) > P.max_velocity || fabs(s.v[1]) > P.max_velocity || fabs(s.v[2]) > P.max_velocity) ok = false;
    if (T < P.min_temp) ok = false;
    if (T > P.max_temp) ok = false;
    return ok;
}

// e4/fvcell.d:975-1059 signal_frequency on a Cartesian structured block
// L: the cell's lengths in the i, j and k directions.
__device__ __forceinline__ double signal_frequency(const NumParams& P, const double* L, const Prim<double>& s) {
    const double iL = L[0], jL = L[1], kL = L[2];
    double signal = 0.0;
    double un_N = fabs(s.v[1]);
    double un_E = fabs(s.v[0]);
    double un_T = (P.dims == 3) ? fabs(s.v[2]) : 0.0;
    if (P.stringent_cfl) {
        double un_max = fmax(un_N, un_E);
        double minLength = fmin(iL, jL);
        if (P.dims == 3) { un_max = fmax(un_max, un_T); minLength = fmin(minLength, kL); }
        signal = (un_max + s.a) / minLength;
    } else {
        double signalN = (un_N + s.a) / jL;
        signal = fmax(signal, signalN);
        double signalE = (un_E + s.a) / iL;
        signal = fmax(signal, signalE);
        if (P.dims == 3) {
            double signalT = (un_T + s.a) / kL;
            signal = fmax(signal, signalT);
        }
    }
    if (P.mhd) {
        double u_mag_sq = s.v[0] * s.v[0] + s.v[1] * s.v[1];
        if (P.dims == 3) u_mag_sq += s.v[2] * s.v[2];
        double u_mag = sqrt(u_mag_sq);
        double B_mag_sq = s.B[0] * s.B[0] + s.B[1] * s.B[1] + s.B[2] * s.B[2];
        double ca2 = B_mag_sq / s.rho;
        double cfast = sqrt(ca2 + s.a * s.a);
        const double L_min = P.dims == 3 ? fmin(fmin(iL, jL), kL) : fmin(iL, jL);
        signal = fmax(signal, (u_mag + cfast) / L_min);
    }
    return signal;
}

}  // namespace gdfv
