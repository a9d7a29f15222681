// fv_oracle.hpp -- CPU restatement of the Eilmer-4 explicit structured-grid
// finite-volume update.  TEST INFRASTRUCTURE ONLY: this code is the checker
// against which the CUDA path is compared; nothing in the product links it.
//
// Every function cites the reference file:line it restates (paths relative to
// the GDTk source tree, e4/ = src/eilmer/).  The numerics are templated on the
// scalar type so the same source serves FP64 runs and the complex-step
// Jacobian-vector product (src/ntypes/complex.d semantics for fabs/fmin/fmax
// and comparisons on the real part).
//
// Geometry: uniform Cartesian blocks.  For axis-aligned faces the reference's
// quad_properties (src/geom/elements/properties.d:97-140) yields
//   i-faces: n=+x t1=+y t2=+z;  j-faces: n=+y t1=+z t2=+x;  k-faces: n=+z t1=+x t2=+y
// (vertex order in e4/sfluidblock.d:737-829) and the frame transforms of
// src/geom/elements/vector3.d:376-400 reduce exactly to these permutations.
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- scalar helpers
using cplx = std::complex<double>;
inline double re(double x) { return x; }
inline double re(const cplx& x) { return x.real(); }
inline double fabs_(double x) { return std::fabs(x); }
// complex.d:944-955: analytic abs keyed on the real part
inline cplx fabs_(const cplx& z) { return (z.real() < 0.0) ? -z : z; }
inline double fmin_(double a, double b) { return std::fmin(a, b); }
inline double fmax_(double a, double b) { return std::fmax(a, b); }
// complex.d:1035-1118
inline cplx fmin_(const cplx& a, const cplx& b) { return (a.real() <= b.real()) ? a : b; }
inline cplx fmax_(const cplx& a, const cplx& b) { return (a.real() >= b.real()) ? a : b; }
inline double sqrt_(double x) { return std::sqrt(x); }
inline cplx sqrt_(const cplx& x) { return std::sqrt(x); }
inline double exp_(double x) { return std::exp(x); }
inline cplx exp_(const cplx& x) { return std::exp(x); }

// ---------------------------------------------------------------- options
enum FluxCalc { FLUX_AUSMDV = 0, FLUX_HLLC = 1, FLUX_HLLE = 2 };
enum Scheme { SCHEME_EULER = 0, SCHEME_PC = 1, SCHEME_TVD_RK3 = 2 };
enum BcType { BC_SLIP_WALL = 0, BC_EXTRAPOLATE = 1, BC_INFLOW = 2, BC_EXCHANGE = 3, BC_FIXED_P = 4, BC_FIXED_PT = 5,
              BC_SIMPLE_FLUX = 6, BC_USER_GHOST = 7 };
enum FaceId { WEST = 0, EAST = 1, SOUTH = 2, NORTH = 3, BOTTOM = 4, TOP = 5 };  // geom nomenclature.d:12-19

// Conserved-quantity indices, e4/conservedquantities.d:148-197 (standard ordering, 3D or MHD)
enum Cqi { MASS = 0, XMOM = 1, YMOM = 2, ZMOM = 3, TOTENERGY = 4, XB = 5, YB = 6, ZB = 7, PSI = 8, DIVB = 9 };

struct Config {
    int flux = FLUX_AUSMDV;
    int scheme = SCHEME_PC;
    int dimensions = 3;
    int mhd = 0;
    int divergence_cleaning = 0;
    int apply_limiter = 1;          // e4/globalconfig.d:1078
    int extrema_clipping = 1;       // :1082
    int apply_entropy_fix = 1;      // :1092
    int glm_reference_indexing = 1; // 1: z-term into F[xB] as e4/fluxcalc.d:146 does
    int stringent_cfl = 0;
    int cfl_count = 10;
    int max_attempts = 3;           // :951
    int max_invalid_cells = 0;      // :1018
    int chicken_compat = 0;         // unit lengths in the limiter and sound speed recomputed (src/chicken)
    int lmr_epsilon = 0;            // van Albada epsilon scaled per face as lmr/onedinterp.d:147-151 does
    double eps_van_albada = 1.0e-12;
    double R = 287.1;
    double gamma = 1.4;
    double cfl = 0.5;
    double dt_init = 1.0e-3;
    double dt_max = 1.0e-3;
    double divB_damping_length = 1.0;
    double max_velocity = 30000.0;  // globalconfig.d:81
    double max_temp = 50000.0;      // :84
    double min_temp = 0.0;          // :85
};

// Ideal gas, src/gas/ideal_gas.d:30-144
struct Gas {
    double R, gamma, Cv, Cvinv, Cp;
    explicit Gas(double R_ = 287.1, double g = 1.4) {
        R = R_; gamma = g;
        Cv = R / (gamma - 1.0);
        Cvinv = 1.0 / Cv;
        Cp = R * gamma / (gamma - 1.0);
    }
};

template <class T>
struct FlowState {
    T rho{0}, p{0}, Tg{0}, u{0}, a{0};
    T vel[3] = {T(0), T(0), T(0)};
    T B[3] = {T(0), T(0), T(0)};
    T psi{0}, divB{0};
};

// ideal_gas.d:98-106.  Returns false where the reference throws GasModelException.
template <class T>
inline bool update_thermo_from_rhou(const Gas& g, FlowState<T>& q) {
    if (re(q.u) <= 0.0 || re(q.rho) <= 0.0) return false;
    q.Tg = q.u * g.Cvinv;
    q.p = q.rho * g.R * q.Tg;
    return true;
}
// ideal_gas.d:107-115
template <class T>
inline bool update_thermo_from_rhoT(const Gas& g, FlowState<T>& q) {
    if (re(q.Tg) <= 0.0 || re(q.rho) <= 0.0) return false;
    q.p = q.rho * g.R * q.Tg;
    q.u = g.Cv * q.Tg;
    return true;
}
// ideal_gas.d:89-97
template <class T>
inline bool update_thermo_from_pT(const Gas& g, FlowState<T>& q) {
    if (re(q.Tg) <= 0.0 || re(q.p) <= 0.0) return false;
    q.rho = q.p / (q.Tg * g.R);
    q.u = g.Cv * q.Tg;
    return true;
}
// ideal_gas.d:132-139
template <class T>
inline bool update_sound_speed(const Gas& g, FlowState<T>& q) {
    if (re(q.Tg) <= 0.0) return false;
    q.a = sqrt_(g.gamma * g.R * q.Tg);
    return true;
}

// ---------------------------------------------------------------- reconstruction
// src/nm/limiters.d:41-50
template <class T>
inline T clip_to_limits(T q, T A, T B) {
    T lower = (re(A) <= re(B)) ? A : B;
    T upper = (re(A) > re(B)) ? A : B;
    T qc = (re(q) > re(lower)) ? q : lower;
    return (re(qc) <= re(upper)) ? qc : upper;
}

// e4/onedinterp.d:338-386 (l2r2_prepare + interp_l2r2_scalar), beta = 1
template <class T>
struct L2R2 {
    T aL0, aR0, lenL0_, lenR0_, two_over_lenL0_plus_lenL1, two_over_lenR0_plus_lenL0,
        two_over_lenR1_plus_lenR0, two_lenL0_plus_lenL1, two_lenR0_plus_lenR1;
    const Config* cfg;
    L2R2(const Config* c, T lenL1, T lenL0, T lenR0, T lenR1) : cfg(c) {
        lenL0_ = lenL0;
        lenR0_ = lenR0;
        aL0 = 0.5 * lenL0 / (lenL1 + 2.0 * lenL0 + lenR0);
        aR0 = 0.5 * lenR0 / (lenL0 + 2.0 * lenR0 + lenR1);
        two_over_lenL0_plus_lenL1 = 2.0 / (lenL0 + lenL1);
        two_over_lenR0_plus_lenL0 = 2.0 / (lenR0 + lenL0);
        two_over_lenR1_plus_lenR0 = 2.0 / (lenR1 + lenR0);
        two_lenL0_plus_lenL1 = (2.0 * lenL0 + lenL1);
        two_lenR0_plus_lenR1 = (2.0 * lenR0 + lenR1);
    }
    void scalar(T qL1, T qL0, T qR0, T qR1, T& qL, T& qR) const {
        T delLminus = (qL0 - qL1) * two_over_lenL0_plus_lenL1;
        T del = (qR0 - qL0) * two_over_lenR0_plus_lenL0;
        T delRplus = (qR1 - qR0) * two_over_lenR1_plus_lenR0;
        T sL = 1.0, sR = 1.0;
        if (cfg->apply_limiter) {
            T eps = cfg->eps_van_albada;
            if (cfg->lmr_epsilon) {
                // lmr/onedinterp.d:147-151: epsilon dimensionalised by the larger of the
                // two states beside the face and the face's length factor
                T qqL = fmax_(T(1e-12), fabs_(qL0));
                T qqR = fmax_(T(1e-12), fabs_(qR0));
                T qq = fmax_(qqL, qqR);
                eps = qq * cfg->eps_van_albada * two_over_lenR0_plus_lenL0;
            }
            sL = (delLminus * del + fabs_(delLminus * del) + eps) / (delLminus * delLminus + del * del + eps);
            sR = (del * delRplus + fabs_(del * delRplus) + eps) / (del * del + delRplus * delRplus + eps);
        }
        const double beta = 1.0;
        qL = qL0 + beta * sL * aL0 * (del * two_lenL0_plus_lenL1 + delLminus * lenR0_);
        qR = qR0 - beta * sR * aR0 * (delRplus * lenL0_ + del * two_lenR0_plus_lenR1);
        if (cfg->extrema_clipping) {
            qL = clip_to_limits(qL, qL0, qR0);
            qR = clip_to_limits(qR, qL0, qR0);
        }
    }
};

// Permutation from global (x,y,z) to the face-local (n,t1,t2) frame for an
// axis-aligned face with normal along axis d.
inline void local_axes(int d, int& an, int& at1, int& at2) {
    an = d; at1 = (d + 1) % 3; at2 = (d + 2) % 3;
}

// e4/onedinterp.d:751-989 (interp_l2r2, thermo_interpolator = rhou, local frame),
// including the copy-on-EOS-failure fallback of :44-74.  Velocities (and B)
// of Lft/Rght come back in the global frame, as in the reference.
template <class T>
void interp_l2r2(const Config& cfg, const Gas& g, int d,
                 const FlowState<T>& cL1, const FlowState<T>& cL0,
                 const FlowState<T>& cR0, const FlowState<T>& cR1,
                 T lenL1, T lenL0, T lenR0, T lenR1,
                 FlowState<T>& Lft, FlowState<T>& Rght) {
    int an, at1, at2;
    local_axes(d, an, at1, at2);
    Lft = cL0;  // onedinterp.d:121-122
    Rght = cR0;
    L2R2<T> w(&cfg, lenL1, lenL0, lenR0, lenR1);
    // velocity in the interface frame
    T vL[3], vR[3];
    const int ax[3] = {an, at1, at2};
    for (int c = 0; c < 3; ++c) {
        int a = ax[c];
        w.scalar(cL1.vel[a], cL0.vel[a], cR0.vel[a], cR1.vel[a], vL[c], vR[c]);
    }
    T BL[3], BR[3];
    if (cfg.mhd) {
        for (int c = 0; c < 3; ++c) {
            int a = ax[c];
            w.scalar(cL1.B[a], cL0.B[a], cR0.B[a], cR1.B[a], BL[c], BR[c]);
        }
        if (cfg.divergence_cleaning) {
            w.scalar(cL1.psi, cL0.psi, cR0.psi, cR1.psi, Lft.psi, Rght.psi);
        }
    }
    w.scalar(cL1.rho, cL0.rho, cR0.rho, cR1.rho, Lft.rho, Rght.rho);
    w.scalar(cL1.u, cL0.u, cR0.u, cR1.u, Lft.u, Rght.u);
    // back to the global frame (exact permutation)
    for (int c = 0; c < 3; ++c) {
        Lft.vel[ax[c]] = vL[c];
        Rght.vel[ax[c]] = vR[c];
        if (cfg.mhd) { Lft.B[ax[c]] = BL[c]; Rght.B[ax[c]] = BR[c]; }
    }
    if (!update_thermo_from_rhou(g, Lft)) { Lft = cL0; }
    if (!update_thermo_from_rhou(g, Rght)) { Rght = cR0; }
    if (cfg.chicken_compat) {
        // chicken's update_from_rhoe recomputes the sound speed (src/chicken/gas.cu:79-85)
        update_sound_speed(g, Lft);
        update_sound_speed(g, Rght);
    }
}

// ---------------------------------------------------------------- flux calculators
// All operate in the interface-local frame: vel[0] = normal component.
// e4/fluxcalc.d:477-651
template <class T>
void ausmdv(const Config& cfg, const Gas& g, const FlowState<T>& L, const FlowState<T>& R, T* F) {
    T rL = L.rho, pL = L.p, pLrL = pL / rL;
    T uL = L.vel[0], vL = L.vel[1], wL = L.vel[2];
    T eL = L.u, aL = L.a;
    T keL = 0.5 * (uL * uL + vL * vL + wL * wL);
    T HL = eL + pLrL + keL;
    T rR = R.rho, pR = R.p, pRrR = pR / rR;
    T uR = R.vel[0], vR = R.vel[1], wR = R.vel[2];
    T eR = R.u, aR = R.a;
    T keR = 0.5 * (uR * uR + vR * vR + wR * wR);
    T HR = eR + pRrR + keR;
    T alphaL = 2.0 * pLrL / (pLrL + pRrR);
    T alphaR = 2.0 * pRrR / (pLrL + pRrR);
    T am = fmax_(aL, aR);
    T ML = uL / am;
    T MR = uR / am;
    T pLplus, uLplus;
    T duL = 0.5 * (uL + fabs_(uL));
    if (re(fabs_(ML)) <= 1.0) {
        pLplus = pL * (ML + 1.0) * (ML + 1.0) * (2.0 - ML) * 0.25;
        uLplus = alphaL * ((uL + am) * (uL + am) / (4.0 * am) - duL) + duL;
    } else {
        pLplus = pL * duL / uL;
        uLplus = duL;
    }
    T pRminus, uRminus;
    T duR = 0.5 * (uR - fabs_(uR));
    if (re(fabs_(MR)) <= 1.0) {
        pRminus = pR * (MR - 1.0) * (MR - 1.0) * (2.0 + MR) * 0.25;
        uRminus = alphaR * (-(uR - am) * (uR - am) / (4.0 * am) - duR) + duR;
    } else {
        pRminus = pR * duR / uR;
        uRminus = duR;
    }
    T ru_half = uLplus * rL + uRminus * rR;
    T p_half = pLplus + pRminus;
    T dp = pL - pR;
    const double K_SWITCH = 10.0;
    dp = K_SWITCH * fabs_(dp) / fmin_(pL, pR);
    T s = 0.5 * fmin_(T(1.0), dp);
    T ru2_AUSMV = uLplus * rL * uL + uRminus * rR * uR;
    T ru2_AUSMD = 0.5 * (ru_half * (uL + uR) - fabs_(ru_half) * (uR - uL));
    T ru2_half = (0.5 + s) * ru2_AUSMV + (0.5 - s) * ru2_AUSMD;
    const double factor = 1.0;
    F[MASS] += factor * ru_half;
    if (re(ru_half) >= 0.0) {
        F[XMOM] += (ru2_half + p_half) * factor;
        F[YMOM] += (ru_half * vL) * factor;
        F[ZMOM] += (ru_half * wL) * factor;
        F[TOTENERGY] += factor * ru_half * HL;
    } else {
        F[XMOM] += (ru2_half + p_half) * factor;
        F[YMOM] += (ru_half * vR) * factor;
        F[ZMOM] += (ru_half * wR) * factor;
        F[TOTENERGY] += factor * ru_half * HR;
    }
    if (cfg.apply_entropy_fix) {
        const double C_EFIX = 0.125;
        bool caseA = (re(uL - aL) < 0.0) && (re(uR - aR) > 0.0);
        bool caseB = (re(uL + aL) < 0.0) && (re(uR + aR) > 0.0);
        T d_ua = 0.0;
        if (caseA && !caseB) { d_ua = C_EFIX * ((uR - aR) - (uL - aL)); }
        if (caseB && !caseA) { d_ua = C_EFIX * ((uR + aR) - (uL + aL)); }
        if (re(d_ua) != 0.0) {
            F[MASS] -= factor * d_ua * (rR - rL);
            F[XMOM] -= factor * d_ua * (rR * uR - rL * uL);
            F[YMOM] -= factor * d_ua * (rR * vR - rL * vL);
            F[ZMOM] -= factor * d_ua * (rR * wR - rL * wL);
            F[TOTENERGY] -= factor * d_ua * (rR * HR - rL * HL);
        }
    }
}

// e4/fluxcalc.d:653-820
template <class T>
void hllc(const Config& cfg, const Gas& g, const FlowState<T>& L, const FlowState<T>& R, T* F) {
    (void)cfg;
    T gL = g.gamma, rL = L.rho, pL = L.p, uL = L.vel[0], vL = L.vel[1], wL = L.vel[2];
    T eL = L.u, aL = L.a;
    T keL = 0.5 * (uL * uL + vL * vL + wL * wL);
    T EL = rL * eL + rL * keL;
    T gR = g.gamma, rR = R.rho, pR = R.p, uR = R.vel[0], vR = R.vel[1], wR = R.vel[2];
    T eR = R.u, aR = R.a;
    T keR = 0.5 * (uR * uR + vR * vR + wR * wR);
    T ER = rR * eR + rR * keR;
    T uhat = (sqrt_(rL) * uL + sqrt_(rR) * uR) / (sqrt_(rL) + sqrt_(rR));
    T ghat = (sqrt_(rL) * gL + sqrt_(rR) * gR) / (sqrt_(rL) + sqrt_(rR));
    T ahat2 = ((sqrt_(rL) * aL * aL + sqrt_(rR) * aR * aR) / (sqrt_(rL) + sqrt_(rR))) +
              0.5 * (ghat - 1.0) * ((sqrt_(rL) + sqrt_(rR)) / sqrt_((sqrt_(rL) + sqrt_(rR)))) * (uR - uL) * (uR - uL);
    T ahat = sqrt_(ahat2);
    T SL = fmin_(uL - aL, uhat - ahat);
    T SR = fmax_(uR + aR, uhat + ahat);
    T S_star = (pR - pL + rL * uL * (SL - uL) - rR * uR * (SR - uR)) / (rL * (SL - uL) - rR * (SR - uR));
    const double factor = 1.0;
    auto flux_fn = [&](bool star, T coeff, T r, T p, T u, T v, T w, T E, T S) {
        T F_mass = r * u;
        T U_mass = r;
        T U_star_mass = coeff;
        T ru_half = star ? F_mass + S * (U_star_mass - U_mass) : F_mass;
        F[MASS] += factor * ru_half;
        T F_momx = r * u * u + p, U_momx = r * u, U_star_momx = coeff * S_star;
        T F_momy = r * u * v, U_momy = r * v, U_star_momy = coeff * v;
        T F_momz = r * u * w, U_momz = r * w, U_star_momz = coeff * w;
        if (star) {
            F[XMOM] += factor * (F_momx + S * (U_star_momx - U_momx));
            F[YMOM] += factor * (F_momy + S * (U_star_momy - U_momy));
            F[ZMOM] += factor * (F_momz + S * (U_star_momz - U_momz));
        } else {
            F[XMOM] += factor * F_momx;
            F[YMOM] += factor * F_momy;
            F[ZMOM] += factor * F_momz;
        }
        T F_totenergy = u * (E + p);
        T U_totenergy = E;
        T U_star_totenergy = coeff * (E / r + (S_star - u) * (S_star + p / (r * (S - u))));
        if (star) F[TOTENERGY] += factor * (F_totenergy + S * (U_star_totenergy - U_totenergy));
        else F[TOTENERGY] += factor * (F_totenergy);
    };
    if (re(S_star) > 0.0) {
        if (re(SL) > 0.0) {
            flux_fn(false, T(0.0), rL, pL, uL, vL, wL, EL, SL);
        } else {
            T coeffL = rL * (SL - uL) / (SL - S_star);
            flux_fn(true, coeffL, rL, pL, uL, vL, wL, EL, SL);
        }
    } else {
        if (re(SR) < 0.0) {
            flux_fn(false, T(0.0), rR, pR, uR, vR, wR, ER, SR);
        } else {
            T coeffR = rR * (SR - uR) / (SR - S_star);
            flux_fn(true, coeffR, rR, pR, uR, vR, wR, ER, SR);
        }
    }
}

// e4/fluxcalc.d:1608-1780 (MHD HLLE, mu0 = 1 units)
template <class T>
void hlle_mhd(const Config& cfg, const Gas& g, const FlowState<T>& L, const FlowState<T>& R, T* F) {
    (void)cfg;
    auto SAFESQRT = [](T x) -> T { return (re(fabs_(x)) > 1.0e-14) ? sqrt_(x) : T(0.0); };
    T rL = L.rho, pL = L.p, uL = L.vel[0], vL = L.vel[1], wL = L.vel[2];
    T BxL = L.B[0], ByL = L.B[1], BzL = L.B[2];
    T rR = R.rho, pR = R.p, uR = R.vel[0], vR = R.vel[1], wR = R.vel[2];
    T BxR = R.B[0], ByR = R.B[1], BzR = R.B[2];
    T cvL = g.Cv, RgasL = g.R, cvR = g.Cv, RgasR = g.R;
    T rLsqrt = sqrt_(rL), rRsqrt = sqrt_(rR);
    T alpha = rLsqrt / (rLsqrt + rRsqrt);
    T cv = alpha * cvL + (1.0 - alpha) * cvR;
    T Rgas = alpha * RgasL + (1.0 - alpha) * RgasR;
    T cp = cv + Rgas;
    T gam = cp / cv;
    T rho = 0.5 * (rL + rR);
    T p = 0.5 * (pL + pR);
    T u = 0.5 * (uL + uR);
    T Bx = 0.5 * (BxL + BxR), By = 0.5 * (ByL + ByR), Bz = 0.5 * (BzL + BzR);
    T a2 = gam * p / rho;
    T Bx2 = Bx * Bx;
    T Bt2 = By * By + Bz * Bz;
    T BB = Bx2 + Bt2;
    T ca2 = Bx2 / rho;
    T alf = a2 + BB / rho;
    T als = SAFESQRT(alf * alf - 4.0 * a2 * ca2);
    T cf2 = 0.5 * (alf + als);
    T cf = sqrt_(cf2);
    T wp = u + cf;
    T wm = u - cf;
    T BxL2 = BxL * BxL, BtL2 = ByL * ByL + BzL * BzL, BBL = BxL2 + BtL2;
    T ptL = pL + 0.5 * BBL;
    T uL2 = uL * uL, uuL = uL2 + vL * vL + wL * wL;
    T aL2 = gam * pL / rL, caL2 = BxL2 / rL, alfL = aL2 + BBL / rL;
    T alsL = SAFESQRT(alfL * alfL - 4.0 * aL2 * caL2);
    T cfL2 = 0.5 * (alfL + alsL), cfL = sqrt_(cfL2);
    T wmL = uL - cfL;
    T BxR2 = BxR * BxR, BtR2 = ByR * ByR + BzR * BzR, BBR = BxR2 + BtR2;
    T ptR = pR + 0.5 * BBR;
    T uR2 = uR * uR, uuR = uR2 + vR * vR + wR * wR;
    T aR2 = gam * pR / rR, caR2 = BxR2 / rR, alfR = aR2 + BBR / rR;
    T alsR = SAFESQRT(alfR * alfR - 4.0 * aR2 * caR2);
    T cfR2 = 0.5 * (alfR + alsR), cfR = sqrt_(cfR2);
    T wpR = uR + cfR;
    T dU[8];
    dU[0] = rR - rL;
    dU[1] = rR * uR - rL * uL;
    dU[2] = rR * vR - rL * vL;
    dU[3] = rR * wR - rL * wL;
    dU[4] = BxR - BxL;
    dU[5] = ByR - ByL;
    dU[6] = BzR - BzL;
    dU[7] = (pR - pL) / (gam - 1.0) + 0.5 * (rR * uuR + BBR) - 0.5 * (rL * uuL + BBL);
    T bl = fmin_(wmL, wm);
    T br = fmax_(wpR, wp);
    T blm = fmin_(bl, T(0.0));
    T brp = fmax_(br, T(0.0));
    T fmassL = rL * uL, fmassR = rR * uR;
    T fmomxL = rL * uL2 - BxL2 + ptL, fmomxR = rR * uR2 - BxR2 + ptR;
    T fmomyL = rL * uL * vL - BxL * ByL, fmomyR = rR * uR * vR - BxR * ByR;
    T fmomzL = rL * uL * wL - BxL * BzL, fmomzR = rR * uR * wR - BxR * BzR;
    T fBxL = 0.0, fBxR = 0.0;
    T fByL = uL * ByL - vL * BxL, fByR = uR * ByR - vR * BxR;
    T fBzL = uL * BzL - wL * BxL, fBzR = uR * BzR - wR * BxR;
    T fenergyL = (rL * L.u + 0.5 * (rL * uuL + BBL) + ptL) * uL - (uL * BxL + vL * ByL + wL * BzL) * BxL;
    T fenergyR = (rR * R.u + 0.5 * (rR * uuR + BBR) + ptR) * uR - (uR * BxR + vR * ByR + wR * BzR) * BxR;
    T iden = 1.0 / (brp - blm);
    T fac1 = brp * blm;
    const double factor = 1.0;
    T mass_flux = factor * (brp * fmassL - blm * fmassR + fac1 * dU[0]) * iden;
    F[MASS] += mass_flux;
    F[XMOM] += factor * ((brp * fmomxL - blm * fmomxR + fac1 * dU[1]) * iden);
    F[YMOM] += factor * ((brp * fmomyL - blm * fmomyR + fac1 * dU[2]) * iden);
    F[ZMOM] += factor * ((brp * fmomzL - blm * fmomzR + fac1 * dU[3]) * iden);
    F[TOTENERGY] += factor * (brp * fenergyL - blm * fenergyR + fac1 * dU[7]) * iden;
    F[XB] += factor * ((brp * fBxL - blm * fBxR + fac1 * dU[4]) * iden);
    F[YB] += factor * ((brp * fByL - blm * fByR + fac1 * dU[5]) * iden);
    F[ZB] += factor * ((brp * fBzL - blm * fBzR + fac1 * dU[6]) * iden);
}

// e4/fluxcalc.d:54-187, compute_interface_flux_interior for a fixed grid
// (gvel = 0, omegaz = 0).  Lft/Rght hold global-frame velocities; F is
// returned in the global frame (F must be zeroed by the caller, fluidblock.d:772).
template <class T>
void interface_flux(const Config& cfg, const Gas& g, double c_h, int d,
                    FlowState<T> Lft, FlowState<T> Rght, T* F) {
    int an, at1, at2;
    local_axes(d, an, at1, at2);
    const int ax[3] = {an, at1, at2};
    FlowState<T> L = Lft, R = Rght;
    for (int c = 0; c < 3; ++c) {
        L.vel[c] = Lft.vel[ax[c]];
        R.vel[c] = Rght.vel[ax[c]];
        if (cfg.mhd) { L.B[c] = Lft.B[ax[c]]; R.B[c] = Rght.B[ax[c]]; }
    }
    switch (cfg.flux) {
    case FLUX_AUSMDV: ausmdv(cfg, g, L, R, F); break;
    case FLUX_HLLC: hllc(cfg, g, L, R, F); break;
    case FLUX_HLLE: hlle_mhd(cfg, g, L, R, F); break;
    }
    if (cfg.mhd) {
        // fluxcalc.d:139-150 (Dedner GLM); the third line targets F[xB] in the reference
        F[DIVB] = 0.5 * (R.B[0] - L.B[0]);
        if (cfg.divergence_cleaning) {
            F[XB] += L.psi + 0.5 * (R.psi - L.psi) - (c_h / 2.0) * (R.B[0] - L.B[0]);
            F[YB] += L.psi + 0.5 * (R.psi - L.psi) - (c_h / 2.0) * (R.B[1] - L.B[1]);
            int zslot = cfg.glm_reference_indexing ? XB : ZB;
            F[zslot] += L.psi + 0.5 * (R.psi - L.psi) - (c_h / 2.0) * (R.B[2] - L.B[2]);
            F[PSI] += (L.B[0] + 0.5 * (R.B[0] - L.B[0]) - (1.0 / (2.0 * c_h)) * (R.psi - L.psi)) * (c_h * c_h);
        }
    }
    // Rotate momentum (and B) fluxes back to the global frame (exact permutation).
    T m[3] = {F[XMOM], F[YMOM], F[ZMOM]};
    for (int c = 0; c < 3; ++c) F[XMOM + ax[c]] = m[c];
    if (cfg.mhd) {
        T b[3] = {F[XB], F[YB], F[ZB]};
        for (int c = 0; c < 3; ++c) F[XB + ax[c]] = b[c];
    }
}

// e4/fvcell.d:511-583 encode_conserved (omegaz = 0, single species)
template <class T>
void encode_conserved(const Config& cfg, const FlowState<T>& fs, T* U) {
    U[MASS] = fs.rho;
    U[XMOM] = fs.rho * fs.vel[0];
    U[YMOM] = fs.rho * fs.vel[1];
    U[ZMOM] = fs.rho * fs.vel[2];
    T u = fs.u;
    T ke = 0.5 * (fs.vel[0] * fs.vel[0] + fs.vel[1] * fs.vel[1] + fs.vel[2] * fs.vel[2]);
    U[TOTENERGY] = fs.rho * (u + ke);
    if (cfg.mhd) {
        U[XB] = fs.B[0]; U[YB] = fs.B[1]; U[ZB] = fs.B[2];
        U[PSI] = fs.psi; U[DIVB] = fs.divB;
        T me = 0.5 * (fs.B[0] * fs.B[0] + fs.B[1] * fs.B[1] + fs.B[2] * fs.B[2]);
        U[TOTENERGY] += me;
    }
}

enum DecodeStatus { DECODE_OK = 0, DECODE_BAD_DENSITY = 1, DECODE_BAD_THERMO = 2 };

// e4/fvcell.d:586-822 decode_conserved; returns where the reference throws.
template <class T>
int decode_conserved(const Config& cfg, const Gas& g, const T* U, FlowState<T>& fs) {
    T rho = U[MASS];
    if (!(re(rho) > 0.0)) return DECODE_BAD_DENSITY;
    fs.rho = rho;
    T dinv = 1.0 / rho;
    fs.vel[0] = U[XMOM] * dinv;
    fs.vel[1] = U[YMOM] * dinv;
    fs.vel[2] = U[ZMOM] * dinv;
    T rE = U[TOTENERGY];
    if (cfg.mhd) {
        fs.B[0] = U[XB]; fs.B[1] = U[YB]; fs.B[2] = U[ZB];
        fs.psi = U[PSI]; fs.divB = U[DIVB];
        T me = 0.5 * (fs.B[0] * fs.B[0] + fs.B[1] * fs.B[1] + fs.B[2] * fs.B[2]);
        rE -= me;
    }
    T u = rE * dinv;
    T ke = 0.5 * (fs.vel[0] * fs.vel[0] + fs.vel[1] * fs.vel[1] + fs.vel[2] * fs.vel[2]);
    u -= ke;
    fs.u = u;
    if (!update_thermo_from_rhou(g, fs)) return DECODE_BAD_THERMO;
    if (re(fs.Tg) <= 0.0) return DECODE_BAD_THERMO;
    if (!update_sound_speed(g, fs)) return DECODE_BAD_THERMO;
    return DECODE_OK;
}

// e4/flowstate.d:363-390 check_data with gas_state.d:226-266
inline bool check_data(const Config& cfg, const FlowState<double>& fs) {
    bool ok = true;
    if (!std::isfinite(fs.rho) || fs.rho < 1.01 * 0.0) ok = false;
    if (!std::isfinite(fs.Tg) || fs.Tg < 1.01 * 0.0) ok = false;
    if (!std::isfinite(fs.p)) ok = false;
    if (!std::isfinite(fs.a)) ok = false;
    if (std::fabs(fs.vel[0]) > cfg.max_velocity || std::fabs(fs.vel[1]) > cfg.max_velocity ||
        std::fabs(fs.vel[2]) > cfg.max_velocity) ok = false;
    if (fs.Tg < cfg.min_temp) ok = false;
    if (fs.Tg > cfg.max_temp) ok = false;
    return ok;
}

// ---------------------------------------------------------------- blocks
struct BoundaryCondition {
    int type = BC_SLIP_WALL;
    int x_order = 0;                 // ExtrapolateCopy xOrder (bc.lua:135)
    int other_block = -1;            // FullFaceCopy partner (full_face_copy.d:65-160)
    int other_face = -1;
    int orientation = 0;             // 0..3 (ignored in 2D)
    bool rotate = false;             // reorient_vector_quantities with Rmatrix R (row major)
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    FlowState<double> inflow;        // FlowStateCopy state
    double p_out = 0.0, T_out = 0.0; // GhostCellFixedP / GhostCellFixedPT (fixed_p.d, fixed_pt.d)
    // UserDefinedGhostCell (e4/bc/ghost_cell_effect/user_defined_effects.d:108-308): ghost
    // states given by the caller, [layer][q][p] over the face (face_extent order)
    std::vector<FlowState<double>> ghost;
};

struct Block {
    int nic = 0, njc = 0, nkc = 0;
    double dx = 1, dy = 1, dz = 1;
    double x0 = 0, y0 = 0, z0 = 0;
    BoundaryCondition bc[6];
    // padded cell arrays: 2 ghost layers on each face
    int pi() const { return nic + 4; }
    int pj() const { return njc + 4; }
    int pk() const { return nkc + 4; }
    size_t ncells() const { return (size_t)nic * njc * nkc; }
    size_t pidx(int i, int j, int k) const {  // i,j,k may be in [-2, n+1]
        return (size_t)(i + 2) + (size_t)pi() * ((size_t)(j + 2) + (size_t)pj() * (size_t)(k + 2));
    }
    size_t cidx(int i, int j, int k) const { return (size_t)i + (size_t)nic * ((size_t)j + (size_t)njc * (size_t)k); }
    std::vector<FlowState<double>> fs;   // padded
    std::vector<double> U[4];            // interior, cell-major: U[l][c*n + q]
    std::vector<double> dUdt[4];
    std::vector<double> Q;               // fixed source term per cell, cell-major (empty: none)
    double length(int d) const { return d == 0 ? dx : (d == 1 ? dy : dz); }
    // Cell lengths per index direction, cells -2 .. n+1 (index c + 2): the block's own cells
    // from its grid, the two ghost layers beyond each face as SFluidBlock gives them
    // (e4/sfluidblock.d:884-1090: ghost n copies the lengths of interior cell n; across a
    // full-face exchange, the partner's cell n, simcore_exchange.d:44-70).  Uniform blocks
    // hold their spacing everywhere.
    bool graded = false;
    std::vector<double> len[3];
    double L(int d, int c) const { return len[d][(size_t)(c + 2)]; }
};

} // namespace orc
