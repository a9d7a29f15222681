// gdfv_stage.cuh -- the fused stage kernel: ghost fill / block exchange,
// l2r2 reconstruction, interface flux, residual assembly, RK stage update,
// decode checks and the CFL signal reduction, in one pass over HBM.
//
// Work decomposition (2.5D blocking): a CTA owns a 32 x TJ column tile of one
// block and marches in k over [k0, k1).  Decoded cell states of the planes
// k, k+1, k+2 sit in a 3-slot shared-memory ring of padded planes (2-cell
// halo in i and j).  Cells outside the block are synthesised by the boundary
// condition of the face they lie beyond (e4/bc/ghost_cell_effect/*), so no
// ghost storage exists in HBM and the inter-block exchange is a direct read
// of the neighbour's conserved state.
//
// Reconstruction is done once per cell and direction: on a uniform grid the
// van Albada limiter that e4/onedinterp.d:357-386 evaluates for the left state
// of face c+1/2 (delLminus, del) and for the right state of face c-1/2
// (del, delRplus) is the same expression of the same two scaled differences,
// so one evaluation gives both interface values of cell c bit for bit.
//
// Per plane: phase A loads the leading plane and the current plane's halo,
// phase B reconstructs (i and j directions through shared memory, k in
// registers of the column's owner thread), phase C evaluates the interface
// fluxes, phase D assembles the residual and the stage update.  The CTA has
// 32*(TJ+1) threads: one per column plus one warp that balances phases B/C.
//
// Stage semantics (e4/simcore_gasdynamic_step.d:1245-1333, predictor-corrector):
//   stage 1: dU0 = R(U0);  U1 = U0 + dt*dU0 is decoded and checked, not stored
//   stage 2: U1 is recomputed on the fly from (U0, dU0) for every loaded cell,
//            dU1 = R(U1);   U2 = U0 + dt*(0.5*dU0 + 0.5*dU1)  -> stored
// giving 5 passes of the state per step.
#pragma once
#include "gdfv_device.cuh"

namespace gdfv {

struct StageArgs {
    const BlockDesc* blocks;
    const TileDesc* tiles;
    const InflowState* inflow;
    double* Ubuf[2];          // conserved state, ping-pong by step parity (SoA [nq][total])
    const double* U_in;       // stage 0 only: explicit input state
    double* dU0;              // stage-1 derivative (SoA)
    double* R_out;            // stage 0: residual output; stage 1 (FP64 flux): predictor state U1 (optional)
    Control* ctl;
    unsigned long long* max_signal;  // per block, bit pattern of a positive double
    double* last_signal;             // per block
    long long total;
    NumParams P;
    int n_tiles;
    int max_invalid_cells;
    int persistent;           // grid of resident CTAs striding over the tiles
    int n_tiles2;             // > 0: the corrector's own tile table follows the first (other rows)
    // Euler kernel of the default options on decoded primitives (gdfv_stage_prim.cuh):
    // primitives (rho, vel, u, a; SoA [6][total], in the flux precision) of Ubuf[0],
    // Ubuf[1] and of the predictor state; null: the stages decode their stencils from the
    // conserved state
    void* prim[2];
    void* prim1;
    // that kernel's own tile tables after the first two (n_tiles + n_tiles2 entries on):
    // n_prim_wide tiles 32 cells wide, then n_prim_narrow tiles 16 wide; both 0: it runs
    // over the first table
    int n_prim_wide, n_prim_narrow;
    // rotations of exchange faces with an Rmatrix (9 doubles each, row major)
    const double* rot;
};

// Compile-time geometry of the tile and of the shared-memory layout.
template <class R, bool MHD, int TJ_>
struct Geo {
    static constexpr int TI = 32, TJ = TJ_;
    // the halo cells of a plane (4 TJ + 4 TI) are one item per thread of the 32 (TJ + 1)
    static_assert(TJ_ >= 4, "column tiles need at least 4 rows");
    static constexpr int NCOL = TI * TJ;
    static constexpr int NT = 32 * (TJ + 1);
    static constexpr int PW = TI + 4, PH = TJ + 4, PLANE = PW * PH;  // padded plane
    static constexpr int NPV = MHD ? 10 : 6;   // rho, v0, v1, v2, u, a, [B0, B1, B2, psi]
    static constexpr int NRS = MHD ? 9 : 5;    // vn, vt1, vt2, rho, u, [Bn, Bt1, Bt2, psi]
    static constexpr int NQ = MHD ? 10 : 5;
    static constexpr int NRI = (TI + 2) * TJ, NRJ = TI * (TJ + 2);
    static constexpr int NFI = (TI + 1) * TJ, NFJ = TI * (TJ + 1);
    static constexpr int O_RING = 0;
    static constexpr int O_RI = O_RING + 3 * NPV * PLANE;
    static constexpr int O_RJ = O_RI + 2 * NRS * NRI;
    static constexpr int O_FI = O_RJ + 2 * NRS * NRJ;
    static constexpr int O_FJ = O_FI + NQ * NFI;
    static constexpr int O_END = O_FJ + NQ * NFJ;
    static constexpr size_t bytes = sizeof(R) * (size_t)O_END;
    // the extra warp takes the first EXTRA items of each flat list, the column threads the rest
    static constexpr int EXTRA = 3 * 32;
};

template <class R>
struct CellR {
    R rho, v[3], u, a, B[3], psi;
};

__device__ __forceinline__ long long cell_index(const BlockDesc& B, int i, int j, int k) {
    return (long long)i + (long long)B.n[0] * ((long long)j + (long long)B.n[1] * (long long)k);
}

// Where the state of block cell (i,j,k) comes from.
enum : int { SRC_CELL = 0, SRC_MIRROR = 1, SRC_EXTRAP1_G0 = 2, SRC_EXTRAP1_G1 = 3, SRC_INFLOW = 4, SRC_FIXEDP = 5,
             SRC_FIXEDPT = 6, SRC_ROTATE = 7 };
struct CellSrc {
    const BlockDesc* blk;  // block holding the source cell(s)
    long long c0, c1;      // source cell (and the depth-1 cell for xOrder 1)
    int kind, axis, inflow;
};

// At most one index may lie outside the block; the boundary condition of that
// face supplies the ghost (e4/bc/ghost_cell_effect/*.d).
// OUTF false: no face of the launch has an OutFlowBC_FixedP, _FixedPT or _SimpleFlux
// boundary (those branches are left out).  ROT false: no exchange face rotates its
// ghosts' vectors (SRC_ROTATE is never returned).
template <bool OUTF = true, bool ROT = true>
__device__ __forceinline__ CellSrc resolve(const StageArgs& A, const BlockDesc& B, int i, int j, int k) {
    CellSrc s;
    s.blk = &B; s.c1 = -1; s.kind = SRC_CELL; s.axis = 0; s.inflow = 0;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    int axis = -1, face = 0, depth = 0;
    if (i < 0) { axis = 0; face = 0; depth = -1 - i; }
    else if (i >= n0) { axis = 0; face = 1; depth = i - n0; }
    else if (j < 0) { axis = 1; face = 2; depth = -1 - j; }
    else if (j >= n1) { axis = 1; face = 3; depth = j - n1; }
    else if (k < 0) { axis = 2; face = 4; depth = -1 - k; }
    else if (k >= n2) { axis = 2; face = 5; depth = k - n2; }
    if (axis < 0) { s.c0 = cell_index(B, i, j, k); return s; }
    s.axis = axis;
    const int type = B.bc_type[face];
    const bool plus = face & 1;
    const int nax = axis == 0 ? n0 : (axis == 1 ? n1 : n2);
    auto at_depth = [&](int m) -> long long {
        int a = plus ? (nax - 1 - m) : m;
        return cell_index(B, axis == 0 ? a : i, axis == 1 ? a : j, axis == 2 ? a : k);
    };
    if (type == BC_SLIP_WALL) {
        s.kind = SRC_MIRROR;            // internal_copy_then_reflect.d:111-150
        s.c0 = at_depth(depth);
    } else if (OUTF && (type == BC_FIXED_P || type == BC_FIXED_PT)) {
        // fixed_p.d:98-119 / fixed_pt.d:105-128: interior cell n with the outside p (T)
        s.kind = type == BC_FIXED_P ? SRC_FIXEDP : SRC_FIXEDPT;
        s.c0 = at_depth(depth);
        s.inflow = B.bc_inflow[face];
    } else if (OUTF && type == BC_SIMPLE_FLUX) {
        s.c0 = at_depth(0);             // its ghosts: ExtrapolateCopy, xOrder 0 (bc.lua:1548)
    } else if (type == BC_EXTRAPOLATE) {
        if (B.bc_xorder[face] == 0) {   // extrapolate_copy.d:124-147
            s.c0 = at_depth(0);
        } else {                        // extrapolate_copy.d:148-168
            s.kind = depth == 0 ? SRC_EXTRAP1_G0 : SRC_EXTRAP1_G1;
            s.c0 = at_depth(0);
            s.c1 = at_depth(1);
        }
    } else if (type == BC_INFLOW) {     // flow_state_copy.d:92-107
        s.kind = SRC_INFLOW;
        s.c0 = -1;
        s.inflow = B.bc_inflow[face];
    } else {
        // full_face_copy.d:680-1409: the partner's cell `depth` layers inside its face,
        // at the tangential position the face pair and orientation give (bc_xlin; 32-bit
        // wrap-around arithmetic, exact since the result is a cell index below 2^31)
        const int* x = B.bc_xlin[face];
        s.blk = &A.blocks[B.bc_other[face]];
        s.c0 = (int)((unsigned)x[0] + (unsigned)x[1] * (unsigned)i + (unsigned)x[2] * (unsigned)j +
                     (unsigned)x[3] * (unsigned)k);
        const int rot = ROT ? B.bc_xrot[face] : 0;
        if (rot) {                      // full_face_copy.d:2403-2405 reorient_vector_quantities
            s.kind = SRC_ROTATE;
            s.inflow = rot - 1;
        }
    }
    return s;
}

// Conserved vector of one cell: stage 2 forms U1 = U0 + dt*dU0 (psi damped).
template <int STAGE, int NQ>
__device__ __forceinline__ void fetch_U(const StageArgs& A, const double* Uin, const BlockDesc& B, long long c,
                                        double dt, double damp, double* U) {
    const long long g = B.offset + c;
#pragma unroll
    for (int q = 0; q < NQ; ++q) U[q] = __ldg(Uin + (long long)q * A.total + g);
    if (STAGE == 2) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) U[q] = d_add(U[q], d_mul(dt, __ldg(A.dU0 + (long long)q * A.total + g)));
        if (NQ == 10 && A.P.divergence_cleaning) U[PSI] = d_mul(U[PSI], damp);
    }
}

// Decode for the state loader.  FAST (FP32-flux variant): the reciprocal of rho
// from a float estimate refined by one FP64 Newton step, and a float square root
// for a, which the float flux arithmetic consumes anyway.  gR = gamma*R.
template <bool FAST, bool MHD>
__device__ __forceinline__ void decode_prim_g(double Cvinv, double gR, const double* U, Prim<double>& s) {
    double rho = U[MASS];
    double dinv;
    if (FAST) {
        double r0 = (double)__frcp_rn((float)rho);
        dinv = r0 * (2.0 - rho * r0);
    } else {
        dinv = 1.0 / rho;
    }
    s.rho = rho;
    s.v[0] = U[XMOM] * dinv;
    s.v[1] = U[YMOM] * dinv;
    s.v[2] = U[ZMOM] * dinv;
    double rE = U[TOTENERGY];
    if (MHD) {
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
    double T = u * Cvinv;
    if (FAST) s.a = (double)sqrtf((float)(gR * T));
    else s.a = sqrt(gR * T);
}

template <bool FAST, bool MHD>
__device__ __forceinline__ void decode_prim(const NumParams& P, const double* U, Prim<double>& s) {
    decode_prim_g<FAST, MHD>(P.gas.Cvinv, P.gas.gamma * P.gas.R, U, s);
}

// flowstate.d:393-400 reorient_vector_quantities: velocity (and B) times the row-major
// matrix R (vector3.d:453-460 apply_matrix_transform, its operation order).  Rare path,
// out of line, with the state passed by value (no caller state needs an address).
template <bool MHD>
__device__ __noinline__ Prim<double> rotate_vectors(const double* R, Prim<double> s) {
    double r[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) r[m] = __ldg(R + m);
    const double x = s.v[0], y = s.v[1], z = s.v[2];
    s.v[0] = d_add(d_add(d_mul(r[0], x), d_mul(r[1], y)), d_mul(r[2], z));
    s.v[1] = d_add(d_add(d_mul(r[3], x), d_mul(r[4], y)), d_mul(r[5], z));
    s.v[2] = d_add(d_add(d_mul(r[6], x), d_mul(r[7], y)), d_mul(r[8], z));
    if (MHD) {
        const double bx = s.B[0], by = s.B[1], bz = s.B[2];
        s.B[0] = d_add(d_add(d_mul(r[0], bx), d_mul(r[1], by)), d_mul(r[2], bz));
        s.B[1] = d_add(d_add(d_mul(r[3], bx), d_mul(r[4], by)), d_mul(r[5], bz));
        s.B[2] = d_add(d_add(d_mul(r[6], bx), d_mul(r[7], by)), d_mul(r[8], bz));
    }
    return s;
}

// extrapolate_copy.d:171-201 linearly_extrapolate_flowstate; fields the
// reference leaves stale (a, psi) come from the boundary cell `edge`.
template <bool MHD>
__device__ __forceinline__ void extrapolate(const Prim<double>& f0, const Prim<double>& f1, const Prim<double>& edge,
                                            Prim<double>& f2) {
    f2 = edge;
    f2.rho = 2.0 * f1.rho - f0.rho;
    f2.u = 2.0 * f1.u - f0.u;
#pragma unroll
    for (int c = 0; c < 3; ++c) f2.v[c] = 2.0 * f1.v[c] - f0.v[c];
    if (MHD) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f2.B[c] = 2.0 * f1.B[c] - f0.B[c];
    }
}

// Ghost of an xOrder=1 extrapolation from the decoded boundary cell e and the
// depth-1 cell at global index g1 (rare path, kept out of line).  Everything
// is passed by value so that no caller state needs an address.
template <int STAGE, bool FAST, bool MHD, int NQ>
__device__ __noinline__ Prim<double> extrap1_ghost(const double* Uin, const double* dU0, long long total, long long g1,
                                                   double dt, double damp, int damp_psi, double Cvinv, double gR,
                                                   Prim<double> e, int depth0) {
    double U1[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) U1[q] = __ldg(Uin + (long long)q * total + g1);
    if (STAGE == 2) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) U1[q] = d_add(U1[q], d_mul(dt, __ldg(dU0 + (long long)q * total + g1)));
        if (NQ == 10 && damp_psi) U1[PSI] = d_mul(U1[PSI], damp);
    }
    Prim<double> f1, g0, out;
    decode_prim_g<FAST, MHD>(Cvinv, gR, U1, f1);
    extrapolate<MHD>(f1, e, e, g0);
    if (depth0) return g0;
    extrapolate<MHD>(e, g0, e, out);
    return out;
}

// Ghost of OutFlowBC_FixedP / _FixedPT from the decoded interior cell e (rare path, out
// of line): update_thermo_from_pT (ideal_gas.d:89-97) with the outside p (and T),
// rho = p/(T R), u = Cv T; velocity and sound speed stay the interior cell's.
static __device__ __noinline__ Prim<double> fixed_ghost(Prim<double> e, bool p_only, double p, double rho_pt, double u_pt,
                                                 double Cvinv, double Cv, double Rg) {
    if (p_only) {
        const double T = e.u * Cvinv;
        e.rho = p / (T * Rg);
        e.u = Cv * T;
    } else {
        e.rho = rho_pt;
        e.u = u_pt;
    }
    return e;
}

template <int STAGE, bool FAST, bool MHD, int NQ, bool OUTF>
__device__ __forceinline__ void finish_cell(const StageArgs& A, const double* Uin, const CellSrc& s,
                                            const double* U0, int i, int j, double dt, double damp,
                                            Prim<double>& out) {
    if (s.kind == SRC_INFLOW) {
        const InflowState& in = A.inflow[s.inflow];
        out.rho = in.rho; out.u = in.u; out.a = in.a; out.psi = in.psi;
        out.v[0] = in.vel[0]; out.v[1] = in.vel[1]; out.v[2] = in.vel[2];
        out.B[0] = in.B[0]; out.B[1] = in.B[1]; out.B[2] = in.B[2];
        return;
    }
    decode_prim<FAST, MHD>(A.P, U0, out);
    if (s.kind == SRC_MIRROR) {
        if (s.axis == 0) out.v[0] = -(out.v[0]);
        else if (s.axis == 1) out.v[1] = -(out.v[1]);
        else out.v[2] = -(out.v[2]);
        if (MHD) {
            // internal_copy_then_reflect.d:140-143 dipole field in slip-wall ghosts with |x| < 0.4136
            const BlockDesc& B = *s.blk;
            double x = B.x0 + ((double)i + 0.5) * B.len[0];
            double y = B.y0 + ((double)j + 0.5) * B.len[1];
            if (x > -0.4136 && x < 0.4136) dipole_field(x, y, out.B[0], out.B[1]);
        }
    } else if (s.kind > SRC_MIRROR) {   // the rare kinds, out of line (SRC_INFLOW returned above)
        if (OUTF && s.kind == SRC_ROTATE) {
            out = rotate_vectors<MHD>(A.rot + 9 * s.inflow, out);
        } else if (OUTF && s.kind >= SRC_FIXEDP) {
            const InflowState& o = A.inflow[s.inflow];
            out = fixed_ghost(out, s.kind == SRC_FIXEDP, o.p, o.rho, o.u, A.P.gas.Cvinv, A.P.gas.Cv, A.P.gas.R);
        } else {
            out = extrap1_ghost<STAGE, FAST, MHD, NQ>(Uin, A.dU0, A.total, s.blk->offset + s.c1, dt, damp,
                                                      A.P.divergence_cleaning, A.P.gas.Cvinv, A.P.gas.gamma * A.P.gas.R,
                                                      out, s.kind == SRC_EXTRAP1_G0);
        }
    }
}

template <class R, int NPV>
__device__ __forceinline__ void put_prim(R* base, int stride, int idx, const Prim<double>& s) {
    base[0 * stride + idx] = (R)s.rho;
    base[1 * stride + idx] = (R)s.v[0];
    base[2 * stride + idx] = (R)s.v[1];
    base[3 * stride + idx] = (R)s.v[2];
    base[4 * stride + idx] = (R)s.u;
    base[5 * stride + idx] = (R)s.a;
    if (NPV > 6) {
        base[6 * stride + idx] = (R)s.B[0];
        base[7 * stride + idx] = (R)s.B[1];
        base[8 * stride + idx] = (R)s.B[2];
        base[9 * stride + idx] = (R)s.psi;
    }
}

template <class R, int NPV>
__device__ __forceinline__ void get_prim(const R* base, int stride, int idx, CellR<R>& c) {
    c.rho = base[0 * stride + idx];
    c.v[0] = base[1 * stride + idx];
    c.v[1] = base[2 * stride + idx];
    c.v[2] = base[3 * stride + idx];
    c.u = base[4 * stride + idx];
    c.a = base[5 * stride + idx];
    if (NPV > 6) {
        c.B[0] = base[6 * stride + idx];
        c.B[1] = base[7 * stride + idx];
        c.B[2] = base[8 * stride + idx];
        c.psi = base[9 * stride + idx];
    } else {
        c.B[0] = c.B[1] = c.B[2] = R(0); c.psi = R(0);
    }
}

// Prim-array variable of reconstructed scalar s in direction D (face-local order
// vn, vt1, vt2, rho, u, Bn, Bt1, Bt2, psi).
template <int D>
__device__ __forceinline__ constexpr int prim_var(int s) {
    return s == 0 ? 1 + D : s == 1 ? 1 + (D + 1) % 3 : s == 2 ? 1 + (D + 2) % 3 : s == 3 ? 0 : s == 4 ? 4
         : s == 5 ? 6 + D : s == 6 ? 6 + (D + 1) % 3 : s == 7 ? 6 + (D + 2) % 3 : 9;
}

// Gather the reconstructed scalars of direction D from a prim array.
template <class R, int NRS, int D>
__device__ __forceinline__ void gather(const R* base, int stride, int idx, R* q) {
#pragma unroll
    for (int s = 0; s < NRS; ++s) q[s] = base[prim_var<D>(s) * stride + idx];
}

// Clip q to the range of A and B (src/nm/limiters.d:41-50).  The FP64 path keeps
// the reference's comparisons; the float path uses min/max (the same value for
// every non-NaN input up to the sign of a zero result).
__device__ __forceinline__ double clip_fast(double q, double A, double B) { return clip_to_limits(q, A, B); }
__device__ __forceinline__ float clip_fast(float q, float A, float B) {
    return fminf(fmaxf(q, fminf(A, B)), fmaxf(A, B));
}

// One cell, one direction: both interface values of every reconstructed scalar
// (e4/onedinterp.d:338-386 with beta = 1 and equal lengths).  qm[s]: value at
// the cell's minus face (right state there), qp[s]: at its plus face (left state).
// psi is reconstructed only with divergence cleaning (onedinterp.d:783-786).
// OPT = 1: apply_limiter and extrema_clipping known to be on (the defaults).
// The float path with OPT = 1 works on raw differences a = q0-qm1, b = qp1-q0
// with the length factors folded into per-direction constants wf (the same
// expressions: dm = a*t, dp = b*t, so the limiter is (ab+|ab|+eps/t^2)/(a^2+b^2+eps/t^2)),
// and without the extrema clipping, which cannot act above float rounding on a
// uniform grid: with equal lengths vp - q0 = sl*(3b + a)/8 and q0 - vm = sl*(b + 3a)/8,
// and sl = (ab + |ab|)/(a^2 + b^2 + e) + e/(a^2 + b^2 + e).  The first part moves vp
// by at most 0.52 b towards qp1 (2ab <= a^2 + b^2, max of 2r(3 + r)/(8(1 + r^2)));
// the second by at most e*m/(2(m^2 + e)) <= sqrt(e)/4, m = max(|a|, |b|), in any
// direction.  So vp leaves [q0, qp1] (vm leaves [qm1, q0]) by at most sqrt(e)/4 =
// 2.5e-7 * cell length, far below float rounding of the reconstructed fields.
enum : int { WF_EPS = 0, WF_P1, WF_P2, WF_R1, WF_R2, WF_N };
template <class R, int NRS, bool MHD, int OPT>
__device__ __forceinline__ void recon_cell(const R* w, const R* wf, const NumParams& P, const R* qm1, const R* q0,
                                           const R* qp1, R* qm, R* qp) {
    if constexpr (sizeof(R) == 4 && OPT == 1) {
        const R e = wf[WF_EPS], P1 = wf[WF_P1], P2 = wf[WF_P2], R1 = wf[WF_R1], R2 = wf[WF_R2];
        // scalars in pairs with packed float2 arithmetic (one instruction per pair),
        // the same operations as the scalar form below
        const float2 e2 = make_float2(e, e), m1 = make_float2(-1.0f, -1.0f);
        const float2 P1v = make_float2(P1, P1), P2v = make_float2(P2, P2);
        const float2 nR1v = make_float2(-R1, -R1), nR2v = make_float2(-R2, -R2);
#pragma unroll
        for (int s = 0; s + 1 < NRS; s += 2) {
            const float2 L = make_float2(qm1[s], qm1[s + 1]), C = make_float2(q0[s], q0[s + 1]);
            const float2 Rr = make_float2(qp1[s], qp1[s + 1]);
            const float2 a = __ffma2_rn(L, m1, C);       // q0 - qm1
            const float2 b = __ffma2_rn(C, m1, Rr);      // qp1 - q0
            const float2 ab = __fmul2_rn(a, b);
            const float2 num = __fadd2_rn(make_float2(ab.x + fabsf(ab.x), ab.y + fabsf(ab.y)), e2);
            const float2 den = __fadd2_rn(__ffma2_rn(b, b, __fmul2_rn(a, a)), e2);
            const float2 sl = __fmul2_rn(num, make_float2(1.0f / den.x, 1.0f / den.y));
            const float2 vp = __ffma2_rn(sl, __ffma2_rn(P1v, b, __fmul2_rn(P2v, a)), C);
            const float2 vm = __ffma2_rn(sl, __ffma2_rn(nR1v, b, __fmul2_rn(nR2v, a)), C);
            qp[s] = vp.x; qp[s + 1] = vp.y;
            qm[s] = vm.x; qm[s + 1] = vm.y;
        }
#pragma unroll
        for (int s = NRS & ~1; s < NRS; ++s) {
            if (MHD && s == 8 && !P.divergence_cleaning) { qm[s] = q0[s]; qp[s] = q0[s]; continue; }
            const R a = q0[s] - qm1[s];
            const R b = qp1[s] - q0[s];
            const R ab = a * b;
            const R sl = (ab + rabs(ab) + e) / (a * a + b * b + e);
            qp[s] = q0[s] + sl * (P1 * b + P2 * a);
            qm[s] = q0[s] - sl * (R1 * b + R2 * a);
        }
    } else {
        const R t = w[W_TOC];
        const R aL0 = w[W_AL0], aR0 = w[W_AR0], len = w[W_LENL0], w3 = w[W_TWOL];
        const bool lim = OPT == 1 ? true : (bool)P.apply_limiter;
        const bool clip = OPT == 1 ? true : (bool)P.extrema_clipping;
        const R eps = R(P.eps_van_albada);
#pragma unroll
        for (int s = 0; s < NRS; ++s) {
            if (MHD && s == 8 && !P.divergence_cleaning) { qm[s] = q0[s]; qp[s] = q0[s]; continue; }
            R dm = (q0[s] - qm1[s]) * t;
            R dp = (qp1[s] - q0[s]) * t;
            R sl = R(1.0), slm = R(1.0);
            if (lim) {
                if (OPT == 0 && P.lmr_epsilon) {
                    // lmr/onedinterp.d:147-151: each face's epsilon is scaled by the larger of
                    // its two states, so the plus face (q0, qp1) and the minus face (qm1, q0)
                    // of the cell get separate limiter values
                    const R tiny = R(1e-12);
                    const R ep = rmax(rmax(tiny, rabs(q0[s])), rmax(tiny, rabs(qp1[s]))) * eps * t;
                    const R em = rmax(rmax(tiny, rabs(qm1[s])), rmax(tiny, rabs(q0[s]))) * eps * t;
                    sl = (dm * dp + rabs(dm * dp) + ep) / (dm * dm + dp * dp + ep);
                    slm = (dm * dp + rabs(dm * dp) + em) / (dm * dm + dp * dp + em);
                } else {
                    sl = (dm * dp + rabs(dm * dp) + eps) / (dm * dm + dp * dp + eps);
                    slm = sl;
                }
            }
            R vp = q0[s] + sl * aL0 * (dp * w3 + dm * len);
            R vm = q0[s] - slm * aR0 * (dp * len + dm * w3);
            if (clip) {
                vp = clip_fast(vp, q0[s], qp1[s]);
                vm = clip_fast(vm, qm1[s], q0[s]);
            }
            qp[s] = vp;
            qm[s] = vm;
        }
    }
}

// recon_cell for a cell of a graded block: the weights g[GW_*] of the cell's position
// along the direction (e4/onedinterp.d:338-386 with the lengths of cells c-1, c, c+1;
// the two scaled differences are those of both faces of the cell, as on a uniform grid).
template <class R, int NRS, bool MHD>
__device__ __forceinline__ void recon_cell_graded(const double* g, const NumParams& P, const R* qm1, const R* q0,
                                                  const R* qp1, R* qm, R* qp) {
    const R tol = R(g[GW_TOL]), toc = R(g[GW_TOC]), a = R(g[GW_A]);
    const R twoL = R(g[GW_TWOL]), lenR0 = R(g[GW_LENR0]), lenL0 = R(g[GW_LENL0]), twoR = R(g[GW_TWOR]);
    const R eps = R(P.eps_van_albada);
#pragma unroll
    for (int s = 0; s < NRS; ++s) {
        if (MHD && s == 8 && !P.divergence_cleaning) { qm[s] = q0[s]; qp[s] = q0[s]; continue; }
        R dm = (q0[s] - qm1[s]) * tol;
        R dp = (qp1[s] - q0[s]) * toc;
        R sl = R(1.0);
        if (P.apply_limiter) sl = (dm * dp + rabs(dm * dp) + eps) / (dm * dm + dp * dp + eps);
        R vp = q0[s] + sl * a * (dp * twoL + dm * lenR0);
        R vm = q0[s] - sl * a * (dp * lenL0 + dm * twoR);
        if (P.extrema_clipping) {
            vp = clip_fast(vp, q0[s], qp1[s]);
            vm = clip_fast(vm, qm1[s], q0[s]);
        }
        qp[s] = vp;
        qm[s] = vm;
    }
}

// AUSMDV (e4/fluxcalc.d:477-651) for the float-flux ideal-gas variant.  The
// ideal-gas identities p/rho = (gamma-1) e and H = e + p/rho + ke = gamma e + ke
// replace the divisions of the general form: alpha = 2 e_L/(e_L + e_R), the
// supersonic pressure split p*du/u is p or 0 by the sign of u.  Velocity
// components are face-local (normal, tangent 1, tangent 2).
__device__ __forceinline__ void ausmdv_f(float g, float gm1, bool efix, float rL, float uL, float vL, float wL,
                                         float eL, float aL, float rR, float uR, float vR, float wR, float eR, float aR,
                                         float* F) {
    // left/right pairs in packed float2 arithmetic where both sides do the same
    const float2 r = make_float2(rL, rR), u = make_float2(uL, uR), v = make_float2(vL, vR);
    const float2 w = make_float2(wL, wR), e = make_float2(eL, eR);
    const float2 p = __fmul2_rn(r, __fmul2_rn(make_float2(gm1, gm1), e));
    const float2 ke = __fmul2_rn(make_float2(0.5f, 0.5f), __ffma2_rn(w, w, __ffma2_rn(v, v, __fmul2_rn(u, u))));
    const float2 H = __ffma2_rn(make_float2(g, g), e, ke);
    const float two_isum = 2.0f / (eL + eR);
    const float2 alpha = __fmul2_rn(e, make_float2(two_isum, two_isum));
    const float am = fmaxf(aL, aR), iam = 1.0f / am;
    const float2 M = __fmul2_rn(u, make_float2(iam, iam));
    const float2 du = __fmul2_rn(make_float2(0.5f, 0.5f), make_float2(uL + fabsf(uL), uR - fabsf(uR)));
    // subsonic splits: p (M +- 1)^2 (2 -+ M)/4 and alpha (Q - du) + du with
    // Q = +-(u +- am)^2 / (4 am)
    const float2 Mo = __fadd2_rn(M, make_float2(1.0f, -1.0f));
    const float2 Mt = __ffma2_rn(M, make_float2(-1.0f, 1.0f), make_float2(2.0f, 2.0f));
    const float2 psub = __fmul2_rn(__fmul2_rn(__fmul2_rn(p, make_float2(0.25f, 0.25f)), __fmul2_rn(Mo, Mo)), Mt);
    const float2 ua = __fadd2_rn(u, make_float2(am, -am));
    const float2 Q = __fmul2_rn(__fmul2_rn(ua, ua), make_float2(0.25f * iam, -0.25f * iam));
    const float2 usub = __ffma2_rn(alpha, __ffma2_rn(du, make_float2(-1.0f, -1.0f), Q), du);
    const bool subL = fabsf(M.x) <= 1.0f, subR = fabsf(M.y) <= 1.0f;
    const float pLplus = subL ? psub.x : (uL > 0.0f ? p.x : 0.0f);
    const float pRminus = subR ? psub.y : (uR < 0.0f ? p.y : 0.0f);
    const float2 us = make_float2(subL ? usub.x : du.x, subR ? usub.y : du.y);
    const float2 ru = __fmul2_rn(us, r);           // (uLplus rL, uRminus rR)
    const float ru_half = ru.x + ru.y;
    const float p_half = pLplus + pRminus;
    const float dp = 10.0f * fabsf(p.x - p.y) / fminf(p.x, p.y);
    const float sw = 0.5f * fminf(1.0f, dp);
    const float2 ruu = __fmul2_rn(ru, u);
    const float ru2_AUSMV = ruu.x + ruu.y;
    const float ru2_AUSMD = 0.5f * (ru_half * (uL + uR) - fabsf(ru_half) * (uR - uL));
    const float ru2_half = (0.5f + sw) * ru2_AUSMV + (0.5f - sw) * ru2_AUSMD;
    const bool up = ru_half >= 0.0f;
    F[0] = ru_half;
    F[1] = ru2_half + p_half;
    F[2] = ru_half * (up ? vL : vR);
    F[3] = ru_half * (up ? wL : wR);
    F[4] = ru_half * (up ? H.x : H.y);
    if (efix) {
        const float C_EFIX = 0.125f;
        const float2 a = make_float2(aL, aR);
        const float2 uma = __ffma2_rn(a, make_float2(-1.0f, -1.0f), u), upa = __fadd2_rn(u, a);
        const bool caseA = (uma.x < 0.0f) && (uma.y > 0.0f);
        const bool caseB = (upa.x < 0.0f) && (upa.y > 0.0f);
        float d_ua = 0.0f;
        if (caseA && !caseB) d_ua = C_EFIX * (uma.y - uma.x);
        if (caseB && !caseA) d_ua = C_EFIX * (upa.y - upa.x);
        if (d_ua != 0.0f) {
            const float2 rv = __fmul2_rn(r, v), rw = __fmul2_rn(r, w), rH = __fmul2_rn(r, H), rU = __fmul2_rn(r, u);
            F[0] -= d_ua * (rR - rL);
            F[1] -= d_ua * (rU.y - rU.x);
            F[2] -= d_ua * (rv.y - rv.x);
            F[3] -= d_ua * (rw.y - rw.x);
            F[4] -= d_ua * (rH.y - rH.x);
        }
    }
}

// boundary_flux_effect.d:504-645 BFE_SimpleOutflowFlux on a fixed Cartesian grid: the
// boundary face (normal +axis D) takes the flux of the interior cell's state (prim
// array pl, entry il) when the mass flux leaves the domain (outsign * m > 0), else the
// face is closed (pressure only).  Fg in the global frame.
template <class R, int D>
__device__ __forceinline__ void simple_outflow_flux(const NumParams& P, const R* pl, int il, int stride, int outsign,
                                                    R* Fg) {
    const R rho = pl[il], u = pl[4 * stride + il];
    const R v[3] = {pl[stride + il], pl[2 * stride + il], pl[3 * stride + il]};
    const R p = rho * R(P.gas.R) * (u * R(P.gas.Cvinv));
    const R nv[3] = {R(D == 0 ? 1.0 : 0.0), R(D == 1 ? 1.0 : 0.0), R(D == 2 ? 1.0 : 0.0)};
    const R vn = v[0] * nv[0] + v[1] * nv[1] + v[2] * nv[2];
    const R m = rho * vn;
    const bool threeD = P.dims == 3;
    if (R(outsign) * m > R(0.0)) {
        Fg[MASS] = m;
        Fg[XMOM] = p * nv[0] + v[0] * m;
        Fg[YMOM] = p * nv[1] + v[1] * m;
        Fg[ZMOM] = threeD ? p * nv[2] + v[2] * m : R(0.0);
        const R utot = u + R(0.5) * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        Fg[TOTENERGY] = m * utot + p * vn;
    } else {
        Fg[MASS] = R(0.0);
        Fg[XMOM] = nv[0] * p;
        Fg[YMOM] = nv[1] * p;
        Fg[ZMOM] = threeD ? nv[2] * p : R(0.0);
        Fg[TOTENERGY] = p * R(0.0);
    }
}

// Interface flux from reconstructed left/right scalars (face-local frame)
// plus the centre states of the two adjacent cells (prim arrays pl/pr, entries
// il/ir, variable stride `stride`): their sound speed is kept (the rhou update
// does not change it) and their full state is the EOS fallback
// (e4/onedinterp.d:44-74), read only when a reconstructed state fails.
// Then compute_interface_flux_interior (e4/fluxcalc.d:54-187) for a fixed grid.
// Fg receives the flux in the global frame.
template <class R, bool MHD, int FLUX, int D, int NPV>
__device__ __forceinline__ void face_flux(const NumParams& P, R c_h, const R* qL, const R* qR, const R* pl, int il,
                                          const R* pr, int ir, int stride, R* Fg) {
    constexpr int NQ = MHD ? 10 : 5;
    constexpr int ax[3] = {D, (D + 1) % 3, (D + 2) % 3};
    if constexpr (sizeof(R) == 4 && !MHD && FLUX == FLUX_AUSMDV) {
        float rL = qL[3], uL = qL[0], vL = qL[1], wL = qL[2], eL = qL[4];
        float rR = qR[3], uR = qR[0], vR = qR[1], wR = qR[2], eR = qR[4];
        if (eL <= 0.0f || rL <= 0.0f) {   // e4/onedinterp.d:44-74: the cell-centre state
            rL = pl[il]; uL = pl[(1 + ax[0]) * stride + il]; vL = pl[(1 + ax[1]) * stride + il];
            wL = pl[(1 + ax[2]) * stride + il]; eL = pl[4 * stride + il];
        }
        if (eR <= 0.0f || rR <= 0.0f) {
            rR = pr[ir]; uR = pr[(1 + ax[0]) * stride + ir]; vR = pr[(1 + ax[1]) * stride + ir];
            wR = pr[(1 + ax[2]) * stride + ir]; eR = pr[4 * stride + ir];
        }
        const float g = (float)P.gas.gamma;
        float F[5];
        ausmdv_f(g, g - 1.0f, P.apply_entropy_fix, rL, uL, vL, wL, eL, pl[5 * stride + il], rR, uR, vR, wR, eR,
                 pr[5 * stride + ir], F);
        Fg[MASS] = F[0];
        Fg[TOTENERGY] = F[4];
#pragma unroll
        for (int m = 0; m < 3; ++m) Fg[XMOM + ax[m]] = F[1 + m];
        return;
    }
    const R Rg = R(P.gas.R), Cvinv = R(P.gas.Cvinv);
    FaceState<R> L, Rr;
    if (qL[4] <= R(0.0) || qL[3] <= R(0.0)) {
        CellR<R> cL;
        get_prim<R, NPV>(pl, stride, il, cL);
        L.rho = cL.rho; L.u = cL.u; L.p = cL.rho * Rg * (cL.u * Cvinv); L.psi = cL.psi;
#pragma unroll
        for (int m = 0; m < 3; ++m) { L.v[m] = cL.v[ax[m]]; L.B[m] = cL.B[ax[m]]; }
    } else {
        L.rho = qL[3]; L.u = qL[4]; L.p = qL[3] * Rg * (qL[4] * Cvinv);
#pragma unroll
        for (int m = 0; m < 3; ++m) { L.v[m] = qL[m]; L.B[m] = MHD ? qL[5 + m] : R(0); }
        L.psi = MHD ? qL[8] : R(0);
    }
    if (qR[4] <= R(0.0) || qR[3] <= R(0.0)) {
        CellR<R> cR;
        get_prim<R, NPV>(pr, stride, ir, cR);
        Rr.rho = cR.rho; Rr.u = cR.u; Rr.p = cR.rho * Rg * (cR.u * Cvinv); Rr.psi = cR.psi;
#pragma unroll
        for (int m = 0; m < 3; ++m) { Rr.v[m] = cR.v[ax[m]]; Rr.B[m] = cR.B[ax[m]]; }
    } else {
        Rr.rho = qR[3]; Rr.u = qR[4]; Rr.p = qR[3] * Rg * (qR[4] * Cvinv);
#pragma unroll
        for (int m = 0; m < 3; ++m) { Rr.v[m] = qR[m]; Rr.B[m] = MHD ? qR[5 + m] : R(0); }
        Rr.psi = MHD ? qR[8] : R(0);
    }
    L.a = pl[5 * stride + il];
    Rr.a = pr[5 * stride + ir];
    R F[NQ];
    if (FLUX == FLUX_AUSMDV) ausmdv(P, L, Rr, F);
    else if (FLUX == FLUX_HLLC) hllc(P, L, Rr, F);
    else hlle_mhd(P, L, Rr, F);
    if (MHD) {
        // fluxcalc.d:139-150; the reference adds the third term to F[xB] (:146)
        F[PSI] = R(0.0);
        F[DIVB] = R(0.5) * (Rr.B[0] - L.B[0]);
        if (P.divergence_cleaning) {
            R pa = L.psi + R(0.5) * (Rr.psi - L.psi);
            F[XB] += pa - (c_h / R(2.0)) * (Rr.B[0] - L.B[0]);
            F[YB] += pa - (c_h / R(2.0)) * (Rr.B[1] - L.B[1]);
            R t3 = pa - (c_h / R(2.0)) * (Rr.B[2] - L.B[2]);
            if (P.glm_reference_indexing) F[XB] += t3; else F[ZB] += t3;
            F[PSI] += (L.B[0] + R(0.5) * (Rr.B[0] - L.B[0]) - (R(1.0) / (R(2.0) * c_h)) * (Rr.psi - L.psi)) * (c_h * c_h);
        }
    }
    Fg[MASS] = F[MASS];
    Fg[TOTENERGY] = F[TOTENERGY];
#pragma unroll
    for (int m = 0; m < 3; ++m) Fg[XMOM + ax[m]] = F[XMOM + m];
    if (MHD) {
#pragma unroll
        for (int m = 0; m < 3; ++m) Fg[XB + ax[m]] = F[XB + m];
        Fg[PSI] = F[PSI];
        Fg[DIVB] = F[DIVB];
    }
}

// Phase-D decode of the float-flux variant: as decode() (e4/fvcell.d:586-822 with
// ideal_gas.d:98-139), with the reciprocal of rho from a float estimate and one
// FP64 Newton step and a float square root for a.  Only the checks and the
// signal frequency consume it; the stored state is the FP64 update itself.
__device__ __forceinline__ int decode_fast(const NumParams& P, const double* U, Prim<double>& s, double& p,
                                           double& T) {
    double rho = U[MASS];
    if (!(rho > 0.0)) return 1;
    s.rho = rho;
    double dinv;
    if (rho > 1.0e-30 && rho < 1.0e30) {
        const double r0 = (double)__frcp_rn((float)rho);
        dinv = r0 * (2.0 - rho * r0);
    } else {
        dinv = 1.0 / rho;
    }
    s.v[0] = U[XMOM] * dinv;
    s.v[1] = U[YMOM] * dinv;
    s.v[2] = U[ZMOM] * dinv;
    s.B[0] = s.B[1] = s.B[2] = 0.0; s.psi = 0.0;
    double u = U[TOTENERGY] * dinv - 0.5 * (s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]);
    s.u = u;
    if (u <= 0.0) return 2;
    T = u * P.gas.Cvinv;
    p = rho * P.gas.R * T;
    if (T <= 0.0) return 2;
    s.a = (double)sqrtf((float)(P.gas.gamma * P.gas.R * T));
    return 0;
}

// signal_frequency (e4/fvcell.d:975-1059) for the float-flux Euler variant with the
// reciprocal cell lengths precomputed (FP64 products instead of divisions).
__device__ __forceinline__ double signal_fast(const NumParams& P, const double* inv_len, const Prim<double>& s) {
    const double un_E = fabs(s.v[0]), un_N = fabs(s.v[1]);
    const double un_T = (P.dims == 3) ? fabs(s.v[2]) : 0.0;
    if (P.stringent_cfl) {
        double un_max = fmax(un_N, un_E);
        double inv_min = fmax(inv_len[0], inv_len[1]);
        if (P.dims == 3) { un_max = fmax(un_max, un_T); inv_min = fmax(inv_min, inv_len[2]); }
        return (un_max + s.a) * inv_min;
    }
    double sig = fmax((un_N + s.a) * inv_len[1], (un_E + s.a) * inv_len[0]);
    if (P.dims == 3) sig = fmax(sig, (un_T + s.a) * inv_len[2]);
    return fmax(sig, 0.0);
}

// Load the state of up to two cells per thread (on[m] says which): resolve, issue
// every global load, then decode (keeps the loads in flight together).  OUTF false:
// no outflow boundary with a rule of its own and no rotating exchange in the launch.
template <int STAGE, bool FAST, bool MHD, int NQ, bool OUTF>
__device__ __forceinline__ void load_two(const StageArgs& A, const double* Uin, const BlockDesc& B, double dt,
                                         double damp, bool on0, bool on1, const int* ci, const int* cj, const int* ck,
                                         Prim<double>* out) {
    CellSrc s[2];
    double U0[2][NQ];
    const bool on[2] = {on0, on1};
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        if (on[m]) {
            s[m] = resolve<OUTF, OUTF>(A, B, ci[m], cj[m], ck[m]);
            if (s[m].kind != SRC_INFLOW) fetch_U<STAGE, NQ>(A, Uin, *s[m].blk, s[m].c0, dt, damp, U0[m]);
        }
    }
#pragma unroll
    for (int m = 0; m < 2; ++m) {
        if (on[m]) finish_cell<STAGE, FAST, MHD, NQ, OUTF>(A, Uin, s[m], U0[m], ci[m], cj[m], dt, damp, out[m]);
    }
}

// Load and decode one cell of the own block at global index g (interior cell: no
// boundary rule applies).
template <int STAGE, bool FAST, bool MHD, int NQ>
__device__ __forceinline__ void load_direct(const StageArgs& A, const double* Uin, long long g, double dt, double damp,
                                            Prim<double>& out) {
    double U[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) U[q] = __ldg(Uin + (long long)q * A.total + g);
    if (STAGE == 2) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) U[q] = d_add(U[q], d_mul(dt, __ldg(A.dU0 + (long long)q * A.total + g)));
        if (NQ == 10 && A.P.divergence_cleaning) U[PSI] = d_mul(U[PSI], damp);
    }
    decode_prim<FAST, MHD>(A.P, U, out);
}

// Resident CTAs per SM the Euler kernels of each flux precision are compiled for
// (register budget; three float-flux CTAs also fill the shared memory).
#ifndef GDFV_MINB_FP32
#define GDFV_MINB_FP32 3
#endif
#ifndef GDFV_MINB_FP64
#define GDFV_MINB_FP64 2
#endif
// MHD kernels: FP64 ones are held to one CTA per SM by their shared memory
#ifndef GDFV_MINB_MHD_FP32
#define GDFV_MINB_MHD_FP32 2
#endif

// PERS = 1: persistent grid over the tile queue; 0: one CTA per tile (no
// state carried between tiles, so the compiler keeps fewer values live).
template <int STAGE, class R, bool MHD, int FLUX, int TJ, int OPT, int PERS>
__global__ void __launch_bounds__(32 * (TJ + 1), MHD ? (sizeof(R) == 4 ? GDFV_MINB_MHD_FP32 : 1)
                                                       : (sizeof(R) == 4 ? GDFV_MINB_FP32 : GDFV_MINB_FP64))
    stage_kernel(StageArgs A) {
    using G = Geo<R, MHD, TJ>;
    constexpr int TI = G::TI, NT = G::NT, NCOL = G::NCOL, PW = G::PW, PLANE = G::PLANE;
    constexpr int NPV = G::NPV, NRS = G::NRS, NQ = G::NQ;
    constexpr int NRI = G::NRI, NRJ = G::NRJ, NFI = G::NFI, NFJ = G::NFJ;
    constexpr bool FAST = sizeof(R) == 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    R* ring = sm + G::O_RING;   // [3][NPV][PLANE]
    R* RI = sm + G::O_RI;       // [2*NRS][NRI]  (q-, q+) per cell, i direction, cells -1..TI
    R* RJ = sm + G::O_RJ;       // [2*NRS][NRJ]  j direction, rows -1..TJ
    R* FI = sm + G::O_FI;       // [NQ][NFI]
    R* FJ = sm + G::O_FJ;       // [NQ][NFJ]
    __shared__ double s_red[NT / 32];
    __shared__ R w[3][W_N];
    __shared__ R wf[3][WF_N];

    const Control* ctl = A.ctl;
    int parity = 0;
    double dt = 0.0;
    if (STAGE != 0) {
        if (ctl->halted || ctl->status != ST_OK) return;
        if (STAGE == 2 && (ctl->n_fail > 0 || ctl->n_invalid1 > A.max_invalid_cells)) return;
        parity = ctl->step & 1;
        dt = ctl->dt_global;
    }
    const double c_h = ctl->c_h;
    const double* Uin = (STAGE == 0) ? A.U_in : A.Ubuf[parity];
    double* Uout = A.Ubuf[parity ^ 1];
    double damp = 1.0;
    if (MHD && A.P.divergence_cleaning && STAGE != 0) {
        // e4/fvcell.d:1068-1074 divergence_damping_factor
        double c_h2 = c_h * c_h;
        double c_p2 = 0.18 * A.P.divB_damping_length * c_h;
        damp = exp(-(c_h2 / c_p2) * dt);
    }

    // Tiles of the block table (ordered by decreasing work).  One CTA per tile, or
    // a persistent grid whose CTAs take tiles from a queue in the control record
    // (one atomic ticket per tile; the last CTA to finish resets the queue).
    __shared__ int s_tile;
    Control* qctl = const_cast<Control*>(ctl);
    int tix = blockIdx.x;
    if (PERS) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(&qctl->tile_next, 1u);
        __syncthreads();
        tix = s_tile;
    }
    while (tix < A.n_tiles) {
        const TileDesc t = A.tiles[tix];
        const int blk = t.block;
        const BlockDesc& B = A.blocks[blk];
        const NumParams& P = A.P;
        const int ni_t = min(TI, B.n[0] - t.i0);
        const int nj_t = min(TJ, B.n[1] - t.j0);
        const int tid = threadIdx.x;
        const bool owner = tid < NCOL;                 // owns column (ti, tj)
        const int ti = tid % TI, tj = tid / TI;
        const bool active = owner && ti < ni_t && tj < nj_t;
        const int pidx = (ti + 2) + PW * (tj + 2);     // own cell in a padded plane
        const bool has_k = (P.dims == 3);
        // faces of this tile on a simple-outflow-flux boundary: bit 2*axis + (plus side);
        // the specialised path (OPT 1) runs only where there are none
        int sfx = 0;
        if (OPT == 0) {
            if (t.i0 == 0 && B.bc_type[0] == BC_SIMPLE_FLUX) sfx |= 1;
            if (t.i0 + ni_t == B.n[0] && B.bc_type[1] == BC_SIMPLE_FLUX) sfx |= 2;
            if (t.j0 == 0 && B.bc_type[2] == BC_SIMPLE_FLUX) sfx |= 4;
            if (t.j0 + nj_t == B.n[1] && B.bc_type[3] == BC_SIMPLE_FLUX) sfx |= 8;
            if (has_k && t.k0 == 0 && B.bc_type[4] == BC_SIMPLE_FLUX) sfx |= 16;
            if (has_k && t.k1 == B.n[2] && B.bc_type[5] == BC_SIMPLE_FLUX) sfx |= 32;
        }
        if (tid < 3 * W_N) w[tid / W_N][tid % W_N] = (R)B.w[tid / W_N][tid % W_N];
        if (tid < 3) {
            const double* bw = B.w[tid];
            const double tc = bw[W_TOC];
            wf[tid][WF_EPS] = (R)(P.eps_van_albada / (tc * tc));
            wf[tid][WF_P1] = (R)(bw[W_AL0] * tc * bw[W_TWOL]);
            wf[tid][WF_P2] = (R)(bw[W_AL0] * tc * bw[W_LENL0]);
            wf[tid][WF_R1] = (R)(bw[W_AR0] * tc * bw[W_LENL0]);
            wf[tid][WF_R2] = (R)(bw[W_AR0] * tc * bw[W_TWOL]);
        }
        const R c_hR = (R)c_h;
        __syncthreads();

        auto slot = [&](int kk) -> R* { return ring + (((kk % 3) + 3) % 3) * NPV * PLANE; };
        // reconstruction of the cell at position pos along direction D (graded blocks take
        // the weights of that position; only the general kernels have graded blocks)
        auto recon = [&](int D, int pos, const R* qm1, const R* q0, const R* qp1, R* qm, R* qp) {
            if (OPT == 0 && B.graded)
                recon_cell_graded<R, NRS, MHD>(B.gw[D] + (pos + 1) * GW_N, P, qm1, q0, qp1, qm, qp);
            else
                recon_cell<R, NRS, MHD, OPT>(w[D], wf[D], P, qm1, q0, qp1, qm, qp);
        };

        R kq_prev_p[NRS];        // k-direction q+ of the current plane (left state of its top face)
        R fB[NQ];                // flux through the bottom face of the owner's cell
#pragma unroll
        for (int q = 0; q < NQ; ++q) fB[q] = R(0);
#pragma unroll
        for (int s = 0; s < NRS; ++s) kq_prev_p[s] = R(0);

        // ---------------- prologue: planes k0-2 .. k0+1 (k0 only in 2D)
        if (has_k) {
            int ci[2] = {t.i0 + ti, t.i0 + ti}, cj[2] = {t.j0 + tj, t.j0 + tj};
            if (active) {
                Prim<double> pr[2];
                int ck[2] = {t.k0 - 2, t.k0 - 1};
                load_two<STAGE, FAST, MHD, NQ, OPT == 0>(A, Uin, B, dt, damp, true, true, ci, cj, ck, pr);
                put_prim<R, NPV>(slot(t.k0 - 2), PLANE, pidx, pr[0]);
                put_prim<R, NPV>(slot(t.k0 - 1), PLANE, pidx, pr[1]);
                int ck2[2] = {t.k0, 0};
                load_two<STAGE, FAST, MHD, NQ, OPT == 0>(A, Uin, B, dt, damp, true, false, ci, cj, ck2, pr);
                put_prim<R, NPV>(slot(t.k0), PLANE, pidx, pr[0]);
                // q+ of plane k0-1 (left state of face k0-1/2); own column only
                R qm1[NRS], q0[NRS], qp1[NRS], qm[NRS];
                gather<R, NRS, 2>(slot(t.k0 - 2), PLANE, pidx, qm1);
                gather<R, NRS, 2>(slot(t.k0 - 1), PLANE, pidx, q0);
                gather<R, NRS, 2>(slot(t.k0), PLANE, pidx, qp1);
                recon(2, t.k0 - 1, qm1, q0, qp1, qm, kq_prev_p);
                // plane k0+1 replaces k0-2 in the ring
                int ck3[2] = {t.k0 + 1, 0};
                load_two<STAGE, FAST, MHD, NQ, OPT == 0>(A, Uin, B, dt, damp, true, false, ci, cj, ck3, pr);
                put_prim<R, NPV>(slot(t.k0 + 1), PLANE, pidx, pr[0]);
                R qkm[NRS], qkp[NRS];
                gather<R, NRS, 2>(slot(t.k0 - 1), PLANE, pidx, qm1);
                gather<R, NRS, 2>(slot(t.k0), PLANE, pidx, q0);
                gather<R, NRS, 2>(slot(t.k0 + 1), PLANE, pidx, qp1);
                recon(2, t.k0, qm1, q0, qp1, qkm, qkp);
                face_flux<R, MHD, FLUX, 2, NPV>(P, c_hR, kq_prev_p, qkm, slot(t.k0 - 1), pidx, slot(t.k0), pidx, PLANE,
                                                fB);
#pragma unroll
                for (int s = 0; s < NRS; ++s) kq_prev_p[s] = qkp[s];
            }
        } else {
            if (active) {
                int ci[2] = {t.i0 + ti, 0}, cj[2] = {t.j0 + tj, 0}, ck[2] = {t.k0, 0};
                Prim<double> pr[2];
                load_two<STAGE, FAST, MHD, NQ, OPT == 0>(A, Uin, B, dt, damp, true, false, ci, cj, ck, pr);
                put_prim<R, NPV>(slot(t.k0), PLANE, pidx, pr[0]);
            }
        }

        double sig_max = 0.0;
        double inv_len[3] = {0.0, 0.0, 0.0};
        if (FAST && !MHD && STAGE == 2) { inv_len[0] = 1.0 / B.len[0]; inv_len[1] = 1.0 / B.len[1]; inv_len[2] = 1.0 / B.len[2]; }
        // halo cell of this thread in every plane (4 columns beside, 4 rows above/below
        // the tile; the extra warp takes items 0..31); the same for all planes
        const int nh = 4 * nj_t + 4 * ni_t;
        const int h = owner ? tid + 32 : tid - NCOL;
        const bool h_on = h < nh;
        int h_ci = 0, h_cj = 0, h_dst = 0;
        if (h_on) {
            int hi, hj;
            if (h < 4 * nj_t) {
                int side = h / (2 * nj_t), rem = h % (2 * nj_t);
                int col = rem / nj_t, row = rem % nj_t;
                hi = side == 0 ? col - 2 : ni_t + col;
                hj = row;
            } else {
                int h2 = h - 4 * nj_t;
                int side = h2 / (2 * ni_t), rem = h2 % (2 * ni_t);
                int row = rem / ni_t, col = rem % ni_t;
                hj = side == 0 ? row - 2 : nj_t + row;
                hi = col;
            }
            h_ci = t.i0 + hi;
            h_cj = t.j0 + hj;
            h_dst = (hi + 2) + PW * (hj + 2);
        }
        // cell indices within the block (32-bit: the host limits a block to 2^31 - 1
        // cells) in plane k of the own cell and of the halo cell when that lies inside
        // the block (no boundary rule), advanced by one plane per step
        const int pstride = B.n[0] * B.n[1];
        int c_own = (t.i0 + ti) + B.n[0] * ((t.j0 + tj) + B.n[1] * t.k0);
        const bool h_in = h_on && h_ci >= 0 && h_ci < B.n[0] && h_cj >= 0 && h_cj < B.n[1];
        int c_halo = (h_in ? h_ci : 0) + B.n[0] * ((h_in ? h_cj : 0) + B.n[1] * t.k0);
        // ring slots of planes k, k+1, k+2
        int r0 = t.k0 % 3;
        const int f0 = owner ? G::EXTRA + tid : tid - NCOL;   // flat-list start and stride
        const int fstride = owner ? NCOL : 32;
        const int fend = owner ? 0x7fffffff : G::EXTRA;

        for (int k = t.k0; k < t.k1; ++k) {
            const int r1 = r0 == 2 ? 0 : r0 + 1, r2 = r1 == 2 ? 0 : r1 + 1;
            R* cur = ring + r0 * (NPV * PLANE);
            R* nx1 = ring + r1 * (NPV * PLANE);
            R* nx2 = ring + r2 * (NPV * PLANE);
            // ---------------- phase A: leading plane k+2 (owners) and the halo of plane k
            {
                const bool lead = active && has_k;
                int ci[2] = {t.i0 + ti, h_ci}, cj[2] = {t.j0 + tj, h_cj}, ck[2] = {k + 2, k};
                // one cell at a time: the FP64 loads and decode of two cells in flight
                // together cost more registers (spills, occupancy) than their overlap gains
                if (lead) {
                    Prim<double> pr[2];
                    if (k + 2 < B.n[2])
                        load_direct<STAGE, FAST, MHD, NQ>(A, Uin, B.offset + (c_own + 2 * pstride), dt, damp, pr[0]);
                    else
                        load_two<STAGE, FAST, MHD, NQ, OPT == 0>(A, Uin, B, dt, damp, true, false, ci, cj, ck, pr);
                    put_prim<R, NPV>(nx2, PLANE, pidx, pr[0]);
                }
                if (h_in) {
                    Prim<double> pr;
                    load_direct<STAGE, FAST, MHD, NQ>(A, Uin, B.offset + c_halo, dt, damp, pr);
                    put_prim<R, NPV>(cur, PLANE, h_dst, pr);
                } else if (h_on) {
                    Prim<double> pr[2];
                    int ci2[2] = {h_ci, 0}, cj2[2] = {h_cj, 0}, ck2[2] = {k, 0};
                    load_two<STAGE, FAST, MHD, NQ, OPT == 0>(A, Uin, B, dt, damp, true, false, ci2, cj2, ck2, pr);
                    put_prim<R, NPV>(cur, PLANE, h_dst, pr[0]);
                }
            }
            __syncthreads();

            // ---------------- phase B: reconstruction
            R kq_m[NRS], kq_p[NRS];
            if (active && has_k) {
                R qm1[NRS], q0[NRS], qp1[NRS];
                gather<R, NRS, 2>(cur, PLANE, pidx, qm1);
                gather<R, NRS, 2>(nx1, PLANE, pidx, q0);
                gather<R, NRS, 2>(nx2, PLANE, pidx, qp1);
                recon(2, k + 1, qm1, q0, qp1, kq_m, kq_p);
            }
            for (int f = f0; f < NRI + NRJ && f < fend; f += fstride) {
                R qm1[NRS], q0[NRS], qp1[NRS], qm[NRS], qp[NRS];
                if (f < NRI) {
                    const int row = f / (TI + 2), ci = f % (TI + 2) - 1;   // cells -1..TI
                    if (row >= nj_t || ci > ni_t) continue;
                    const int p = (ci + 2) + PW * (row + 2);
                    gather<R, NRS, 0>(cur, PLANE, p - 1, qm1);
                    gather<R, NRS, 0>(cur, PLANE, p, q0);
                    gather<R, NRS, 0>(cur, PLANE, p + 1, qp1);
                    recon(0, t.i0 + ci, qm1, q0, qp1, qm, qp);
#pragma unroll
                    for (int s = 0; s < NRS; ++s) { RI[s * NRI + f] = qm[s]; RI[(NRS + s) * NRI + f] = qp[s]; }
                } else {
                    const int g = f - NRI;
                    const int cj = g / TI - 1, col = g % TI;               // rows -1..TJ
                    if (col >= ni_t || cj > nj_t) continue;
                    const int p = (col + 2) + PW * (cj + 2);
                    gather<R, NRS, 1>(cur, PLANE, p - PW, qm1);
                    gather<R, NRS, 1>(cur, PLANE, p, q0);
                    gather<R, NRS, 1>(cur, PLANE, p + PW, qp1);
                    recon(1, t.j0 + cj, qm1, q0, qp1, qm, qp);
#pragma unroll
                    for (int s = 0; s < NRS; ++s) { RJ[s * NRJ + g] = qm[s]; RJ[(NRS + s) * NRJ + g] = qp[s]; }
                }
            }
            __syncthreads();

            // ---------------- phase C: interface fluxes
            R fT[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) fT[q] = R(0);
            if (active && has_k) {
                face_flux<R, MHD, FLUX, 2, NPV>(P, c_hR, kq_prev_p, kq_m, cur, pidx, nx1, pidx, PLANE, fT);
#pragma unroll
                for (int s = 0; s < NRS; ++s) kq_prev_p[s] = kq_p[s];
            }
            for (int f = f0; f < NFI + NFJ && f < fend; f += fstride) {
                R qL[NRS], qR[NRS], F[NQ];
                if (f < NFI) {
                    const int row = f / (TI + 1), fi = f % (TI + 1);       // faces 0..TI
                    if (row >= nj_t || fi > ni_t) continue;
                    const int rl = fi + (TI + 2) * row;                    // RI index of cell fi-1
#pragma unroll
                    for (int s = 0; s < NRS; ++s) { qL[s] = RI[(NRS + s) * NRI + rl]; qR[s] = RI[s * NRI + rl + 1]; }
                    const int p = (fi + 2) + PW * (row + 2);
                    face_flux<R, MHD, FLUX, 0, NPV>(P, c_hR, qL, qR, cur, p - 1, cur, p, PLANE, F);
#pragma unroll
                    for (int q = 0; q < NQ; ++q) FI[q * NFI + f] = F[q];
                } else {
                    const int g = f - NFI;
                    const int fj = g / TI, col = g % TI;                   // faces 0..TJ
                    if (col >= ni_t || fj > nj_t) continue;
                    const int rl = col + TI * fj;                          // RJ index of row fj-1
#pragma unroll
                    for (int s = 0; s < NRS; ++s) { qL[s] = RJ[(NRS + s) * NRJ + rl]; qR[s] = RJ[s * NRJ + rl + TI]; }
                    const int p = (col + 2) + PW * (fj + 2);
                    face_flux<R, MHD, FLUX, 1, NPV>(P, c_hR, qL, qR, cur, p - PW, cur, p, PLANE, F);
#pragma unroll
                    for (int q = 0; q < NQ; ++q) FJ[q * NFJ + g] = F[q];
                }
            }
            __syncthreads();

            // ---------------- boundary faces with OutFlowBC_SimpleFlux (only tiles that have
            // them): their flux is the interior cell's (boundary_flux_effect.d:504-645)
            if (OPT == 0 && sfx) {
                if (active && has_k) {
                    if ((sfx & 16) && k == 0) simple_outflow_flux<R, 2>(P, cur, pidx, PLANE, -1, fB);
                    if ((sfx & 32) && k + 1 == B.n[2]) simple_outflow_flux<R, 2>(P, cur, pidx, PLANE, 1, fT);
                }
                for (int e = tid; e < 2 * nj_t + 2 * ni_t; e += NT) {
                    R F[NQ];
                    if (e < 2 * nj_t) {             // i faces 0 (west) and ni_t (east) of row e / 2
                        const int row = e >> 1, east = e & 1;
                        if (!(sfx & (east ? 2 : 1))) continue;
                        const int fi = east ? ni_t : 0;
                        const int p = (fi + 2) + PW * (row + 2);
                        simple_outflow_flux<R, 0>(P, cur, east ? p - 1 : p, PLANE, east ? 1 : -1, F);
#pragma unroll
                        for (int q = 0; q < NQ; ++q) FI[q * NFI + row * (TI + 1) + fi] = F[q];
                    } else {                        // j faces 0 (south) and nj_t (north) of a column
                        const int col = (e - 2 * nj_t) >> 1, north = (e - 2 * nj_t) & 1;
                        if (!(sfx & (north ? 8 : 4))) continue;
                        const int fj = north ? nj_t : 0;
                        const int p = (col + 2) + PW * (fj + 2);
                        simple_outflow_flux<R, 1>(P, cur, north ? p - PW : p, PLANE, north ? 1 : -1, F);
#pragma unroll
                        for (int q = 0; q < NQ; ++q) FJ[q * NFJ + fj * TI + col] = F[q];
                    }
                }
                __syncthreads();
            }

            // ---------------- phase D: residual (e4/fvcell.d:824-856, faces W, E, S, N, B, T) and update
            if (active) {
                const long long g = B.offset + c_own;
                double dU[NQ];
                double Ai = B.area[0], Aj = B.area[1], Ak = B.area[2], vol_inv = B.vol_inv;
                double clen[3] = {B.len[0], B.len[1], B.len[2]};
                if (OPT == 0 && B.graded) {
                    // face areas and volume of the own cell from its lengths (uniform: dy dz,
                    // dz dx, dx dy and 1/(dx dy dz) as the block's own)
                    cell_lengths(B, t.i0 + ti, t.j0 + tj, k, clen);
                    if (has_k) {
                        Ai = d_mul(clen[1], clen[2]); Aj = d_mul(clen[2], clen[0]); Ak = d_mul(clen[0], clen[1]);
                        vol_inv = 1.0 / d_mul(d_mul(clen[0], clen[1]), clen[2]);
                    } else {
                        Ai = clen[1]; Aj = clen[0];
                        vol_inv = 1.0 / d_mul(clen[0], clen[1]);
                    }
                }
                if (FAST) {
                    // float path: differences of opposite faces in float (same-signed,
                    // nearly equal fluxes subtract exactly), accumulation in FP64
                    const double Vi = vol_inv;
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        R dI = FI[q * NFI + ti + (TI + 1) * tj] - FI[q * NFI + ti + 1 + (TI + 1) * tj];
                        R dJ = FJ[q * NFJ + ti + TI * tj] - FJ[q * NFJ + ti + TI * (tj + 1)];
                        double si = (double)dI * Ai + (double)dJ * Aj;
                        if (has_k) si += (double)(fB[q] - fT[q]) * Ak;
                        dU[q] = Vi * si;
                    }
                } else
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    double FW = (double)FI[q * NFI + ti + (TI + 1) * tj];
                    double FE = (double)FI[q * NFI + ti + 1 + (TI + 1) * tj];
                    double FS = (double)FJ[q * NFJ + ti + TI * tj];
                    double FN = (double)FJ[q * NFJ + ti + TI * (tj + 1)];
                    double si = 0.0;
                    si = __dsub_rn(si, d_mul(FW, -Ai));
                    si = __dsub_rn(si, d_mul(FE, Ai));
                    si = __dsub_rn(si, d_mul(FS, -Aj));
                    si = __dsub_rn(si, d_mul(FN, Aj));
                    if (has_k) {
                        si = __dsub_rn(si, d_mul((double)fB[q], -Ak));
                        si = __dsub_rn(si, d_mul((double)fT[q], Ak));
                    }
                    dU[q] = d_add(d_mul(vol_inv, si), 0.0);
                }
                if (STAGE == 0) {
#pragma unroll
                    for (int q = 0; q < NQ; ++q) A.R_out[(long long)q * A.total + g] = dU[q];
                } else {
                    double U[10];
#pragma unroll
                    for (int q = 0; q < NQ; ++q) U[q] = __ldg(Uin + (long long)q * A.total + g);
                    if (STAGE == 1) {
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            A.dU0[(long long)q * A.total + g] = dU[q];
                            U[q] = d_add(U[q], d_mul(dt, dU[q]));
                        }
                        if (sizeof(R) == 8 && A.R_out) {   // U1 before the psi damping (FP64 adjoint recomputation)
#pragma unroll
                            for (int q = 0; q < NQ; ++q) A.R_out[(long long)q * A.total + g] = U[q];
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            double d0 = __ldg(A.dU0 + (long long)q * A.total + g);
                            U[q] = d_add(U[q], d_mul(dt, d_add(d_mul(0.5, d0), d_mul(0.5, dU[q]))));
                        }
                    }
                    if (MHD && P.divergence_cleaning) U[PSI] = d_mul(U[PSI], damp);
                    if (STAGE == 2) {
#pragma unroll
                        for (int q = 0; q < NQ; ++q) Uout[(long long)q * A.total + g] = U[q];
                    }
                    Prim<double> s;
                    double p, T;
                    int st = (FAST && !MHD) ? decode_fast(P, U, s, p, T) : decode(P, U, s, p, T);
                    if (st != 0) {
                        atomicAdd(&A.ctl->n_fail, 1);
                        atomicMin(reinterpret_cast<unsigned long long*>(&A.ctl->first_bad_cell),
                                  (unsigned long long)g);
                    } else {
                        if (!check_data(P, s, p, T)) {
                            atomicAdd(STAGE == 1 ? &A.ctl->n_invalid1 : &A.ctl->n_invalid2, 1);
                            atomicMin(reinterpret_cast<unsigned long long*>(&A.ctl->first_bad_cell),
                                      (unsigned long long)g);
                        }
                        if (STAGE == 2) {
                            if (FAST && !MHD && OPT == 0 && B.graded) {
                                inv_len[0] = 1.0 / clen[0]; inv_len[1] = 1.0 / clen[1]; inv_len[2] = 1.0 / clen[2];
                            }
                            double sig = (FAST && !MHD) ? signal_fast(P, inv_len, s) : signal_frequency(P, clen, s);
                            sig_max = fmax(sig_max, sig);
                            if (c_own == pstride * B.n[2] - 1) A.last_signal[blk] = sig;
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < NQ; ++q) fB[q] = fT[q];
            c_own += pstride;
            c_halo += pstride;
            r0 = r1;
        }

        if (STAGE == 2) {
            // CTA max of the signal frequency -> one atomic per CTA (dt rule input)
            for (int o = 16; o > 0; o >>= 1) sig_max = fmax(sig_max, __shfl_xor_sync(0xffffffffu, sig_max, o));
            if ((tid & 31) == 0) s_red[tid >> 5] = sig_max;
            __syncthreads();
            if (tid == 0) {
                double m = s_red[0];
                for (int wv = 1; wv < NT / 32; ++wv) m = fmax(m, s_red[wv]);
                atomicMax(&A.max_signal[blk], (unsigned long long)__double_as_longlong(m));
            }
        }
        if (!PERS) break;
        __syncthreads();
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(&qctl->tile_next, 1u);
        __syncthreads();
        tix = s_tile;
    }
    if (PERS && threadIdx.x == 0) {
        // every CTA has taken its last ticket before it counts itself done
        if (atomicAdd(&qctl->tile_done, 1u) == gridDim.x - 1) {
            atomicExch(&qctl->tile_next, 0u);
            atomicExch(&qctl->tile_done, 0u);
        }
    }
}

}  // namespace gdfv
