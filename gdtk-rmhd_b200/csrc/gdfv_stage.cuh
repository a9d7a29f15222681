// gdfv_stage.cuh -- the fused stage kernel: ghost fill / block exchange,
// l2r2 reconstruction, interface flux, residual assembly, RK stage update,
// decode checks and the CFL signal reduction, in one pass over HBM.
//
// Work decomposition (2.5D blocking): a CTA owns a TI x TJ column tile of one
// block and marches in k over [k0, k1).  Decoded cell states live in a
// 4-plane shared-memory ring (planes k-1..k+2 for the k-faces) plus a
// cross-shaped halo for the current plane (x/y neighbours for the i- and
// j-faces).  Cells outside the block are synthesised by the boundary
// condition of the face they lie beyond (e4/bc/ghost_cell_effect/*), so no
// ghost storage exists in HBM and the inter-block exchange is a direct read of
// the neighbour's conserved state.
//
// Stage semantics (e4/simcore_gasdynamic_step.d:1245-1333, predictor-corrector):
//   stage 1: dU0 = R(U0);  U1 = U0 + dt*dU0 is decoded and checked, not stored
//   stage 2: U1 is recomputed on the fly from (U0, dU0) for every loaded cell,
//            dU1 = R(U1);   U2 = U0 + dt*(0.5*dU0 + 0.5*dU1)  -> stored
// giving 5 passes of the state per step.  The update arithmetic is written
// with round-to-nearest intrinsics so that it is not contracted into FMAs.
#pragma once
#include "gdfv_device.cuh"

namespace gdfv {

constexpr int TI = 32;
constexpr int TJ = 8;
constexpr int NT = TI * TJ;
constexpr int NHALO = 4 * TJ + 4 * TI;

struct StageArgs {
    const BlockDesc* blocks;
    const TileDesc* tiles;
    const InflowState* inflow;
    double* Ubuf[2];          // conserved state, ping-pong by step parity (SoA [nq][total])
    const double* U_in;       // stage 0 only: explicit input state
    double* dU0;              // stage-1 derivative (SoA)
    double* R_out;            // stage 0 only: residual output
    Control* ctl;
    unsigned long long* max_signal;  // per block, bit pattern of a positive double
    double* last_signal;             // per block
    long long total;
    NumParams P;
    int n_tiles;
    int max_invalid_cells;
};

template <class R>
struct CellR {
    R rho, v[3], u, a, B[3], psi;
};

__device__ __forceinline__ long long cell_index(const BlockDesc& B, int i, int j, int k) {
    return (long long)i + (long long)B.n[0] * ((long long)j + (long long)B.n[1] * (long long)k);
}

// Read the conserved vector of one cell (stage 2: U1 = U0 + dt*dU0, psi damped) and decode it.
template <int STAGE>
__device__ __forceinline__ int fetch_decode(const StageArgs& A, const double* Uin, const BlockDesc& B,
                                            long long cell, double dt, double damp, Prim<double>& s) {
    const int nq = A.P.nq;
    double U[10];
    const long long g = B.offset + cell;
#pragma unroll
    for (int q = 0; q < 10; ++q) {
        if (q < nq) U[q] = __ldg(Uin + (long long)q * A.total + g);
    }
    if (STAGE == 2) {
#pragma unroll
        for (int q = 0; q < 10; ++q) {
            if (q < nq) U[q] = d_add(U[q], d_mul(dt, __ldg(A.dU0 + (long long)q * A.total + g)));
        }
        if (A.P.mhd && A.P.divergence_cleaning) U[PSI] = d_mul(U[PSI], damp);
    }
    double p, T;
    return decode(A.P, U, s, p, T);
}

// extrapolate_copy.d:171-201 linearly_extrapolate_flowstate; fields the
// reference leaves stale (a, psi) come from the boundary cell `edge`.
__device__ __forceinline__ void extrapolate(const NumParams& P, const Prim<double>& f0, const Prim<double>& f1,
                                            const Prim<double>& edge, Prim<double>& f2) {
    f2 = edge;
    f2.rho = 2.0 * f1.rho - f0.rho;
    f2.u = 2.0 * f1.u - f0.u;
#pragma unroll
    for (int c = 0; c < 3; ++c) f2.v[c] = 2.0 * f1.v[c] - f0.v[c];
    if (P.mhd) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f2.B[c] = 2.0 * f1.B[c] - f0.B[c];
    }
}

// Flow state of block cell (i,j,k); at most one index may lie outside the block,
// in which case the boundary condition of that face supplies a ghost state.
__device__ __forceinline__ void negate_axis(Prim<double>& s, int axis) {
    if (axis == 0) s.v[0] = -(s.v[0]);
    else if (axis == 1) s.v[1] = -(s.v[1]);
    else s.v[2] = -(s.v[2]);
}

// Flow state of block cell (i,j,k); at most one index may lie outside the block,
// in which case the boundary condition of that face supplies a ghost state.
template <int STAGE>
__device__ Prim<double> load_cell(const StageArgs& A, const double* Uin, int blk, int i, int j, int k,
                                  double dt, double damp) {
    const BlockDesc& B = A.blocks[blk];
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    int axis = -1, face = 0, depth = 0;
    if (i < 0) { axis = 0; face = 0; depth = -1 - i; }
    else if (i >= n0) { axis = 0; face = 1; depth = i - n0; }
    else if (j < 0) { axis = 1; face = 2; depth = -1 - j; }
    else if (j >= n1) { axis = 1; face = 3; depth = j - n1; }
    else if (k < 0) { axis = 2; face = 4; depth = -1 - k; }
    else if (k >= n2) { axis = 2; face = 5; depth = k - n2; }
    Prim<double> s;
    if (axis < 0) {
        fetch_decode<STAGE>(A, Uin, B, cell_index(B, i, j, k), dt, damp, s);
        return s;
    }
    const int type = B.bc_type[face];
    const bool plus = face & 1;
    // index of the interior cell at depth m from this face, same cross indices
    auto at_depth = [&](int m) -> long long {
        int a = plus ? (B.n[axis] - 1 - m) : m;
        return cell_index(B, axis == 0 ? a : i, axis == 1 ? a : j, axis == 2 ? a : k);
    };
    if (type == BC_SLIP_WALL) {
        // internal_copy_then_reflect.d:111-150: mirror cell n into ghost n, negate normal velocity
        fetch_decode<STAGE>(A, Uin, B, at_depth(depth), dt, damp, s);
        negate_axis(s, axis);
        if (A.P.mhd) {
            // :140-143 dipole field written into slip-wall ghosts with |x| < 0.4136
            double x = B.x0 + ((double)i + 0.5) * B.len[0];
            double y = B.y0 + ((double)j + 0.5) * B.len[1];
            if (x > -0.4136 && x < 0.4136) {
                double r = pow(pow(pow(x + 0., 2.0) + pow(y + 0.0, 2.0), 0.5), 5.0);
                double cc = ((0.1) * pow(0.82 / 2, 3.0)) / (2 * r);
                s.B[0] = -cc * (2 * pow(x + 0., 2.0) - pow(y + 0.0, 2.0));
                s.B[1] = -cc * (3 * (x + 0.) * (y + 0.0));
            }
        }
    } else if (type == BC_EXTRAPOLATE) {
        if (B.bc_xorder[face] == 0) {
            fetch_decode<STAGE>(A, Uin, B, at_depth(0), dt, damp, s);  // extrapolate_copy.d:124-147
        } else {
            Prim<double> e, f1, g0;
            fetch_decode<STAGE>(A, Uin, B, at_depth(0), dt, damp, e);
            fetch_decode<STAGE>(A, Uin, B, at_depth(1), dt, damp, f1);
            extrapolate(A.P, f1, e, e, g0);
            if (depth == 0) s = g0;
            else extrapolate(A.P, e, g0, e, s);
        }
    } else if (type == BC_INFLOW) {
        const InflowState& in = A.inflow[B.bc_inflow[face]];
        s.rho = in.rho; s.u = in.u; s.a = in.a; s.psi = in.psi;
        s.v[0] = in.vel[0]; s.v[1] = in.vel[1]; s.v[2] = in.vel[2];
        s.B[0] = in.B[0]; s.B[1] = in.B[1]; s.B[2] = in.B[2];
    } else {
        // full_face_copy.d: ghost n <- the partner block's interior cell n from its face
        const BlockDesc& O = A.blocks[B.bc_other[face]];
        const int of = B.bc_other_face[face];
        int a = (of & 1) ? (O.n[axis] - 1 - depth) : depth;
        fetch_decode<STAGE>(A, Uin, O, cell_index(O, axis == 0 ? a : i, axis == 1 ? a : j, axis == 2 ? a : k),
                            dt, damp, s);
    }
    return s;
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

// One interface: l2r2 reconstruction (e4/onedinterp.d:751-989, rhou, local
// frame, EOS fallback of :44-74), then compute_interface_flux_interior
// (e4/fluxcalc.d:54-187) for a fixed grid.  Fg receives the flux in the
// global frame.
template <class R, bool MHD, int FLUX, int D>
__device__ __forceinline__ void face_flux(const NumParams& P, const R* w, R c_h,
                                          const CellR<R>& c1, const CellR<R>& c0, const CellR<R>& d0,
                                          const CellR<R>& d1, R* Fg) {
    constexpr int NQ = MHD ? 10 : 5;
    constexpr int ax[3] = {D, (D + 1) % 3, (D + 2) % 3};
    FaceState<R> L, Rr;
    R vL[3], vR[3], BL[3], BR[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) l2r2(w, P, c1.v[ax[m]], c0.v[ax[m]], d0.v[ax[m]], d1.v[ax[m]], vL[m], vR[m]);
    L.psi = c0.psi; Rr.psi = d0.psi;
    if (MHD) {
#pragma unroll
        for (int m = 0; m < 3; ++m) l2r2(w, P, c1.B[ax[m]], c0.B[ax[m]], d0.B[ax[m]], d1.B[ax[m]], BL[m], BR[m]);
        if (P.divergence_cleaning) l2r2(w, P, c1.psi, c0.psi, d0.psi, d1.psi, L.psi, Rr.psi);
    }
    R rL, rR, uL, uR;
    l2r2(w, P, c1.rho, c0.rho, d0.rho, d1.rho, rL, rR);
    l2r2(w, P, c1.u, c0.u, d0.u, d1.u, uL, uR);
    const R Rg = R(P.gas.R), Cvinv = R(P.gas.Cvinv);
    // update_thermo_from_rhou, falling back to the cell-centre state on failure
    if (uL <= R(0.0) || rL <= R(0.0)) {
        L.rho = c0.rho; L.u = c0.u; L.p = c0.rho * Rg * (c0.u * Cvinv); L.psi = c0.psi;
#pragma unroll
        for (int m = 0; m < 3; ++m) { L.v[m] = c0.v[ax[m]]; L.B[m] = c0.B[ax[m]]; }
    } else {
        L.rho = rL; L.u = uL; L.p = rL * Rg * (uL * Cvinv);
#pragma unroll
        for (int m = 0; m < 3; ++m) { L.v[m] = vL[m]; L.B[m] = MHD ? BL[m] : R(0); }
    }
    if (uR <= R(0.0) || rR <= R(0.0)) {
        Rr.rho = d0.rho; Rr.u = d0.u; Rr.p = d0.rho * Rg * (d0.u * Cvinv); Rr.psi = d0.psi;
#pragma unroll
        for (int m = 0; m < 3; ++m) { Rr.v[m] = d0.v[ax[m]]; Rr.B[m] = d0.B[ax[m]]; }
    } else {
        Rr.rho = rR; Rr.u = uR; Rr.p = rR * Rg * (uR * Cvinv);
#pragma unroll
        for (int m = 0; m < 3; ++m) { Rr.v[m] = vR[m]; Rr.B[m] = MHD ? BR[m] : R(0); }
    }
    L.a = c0.a;   // the rhou update leaves the cell-centre sound speed in place
    Rr.a = d0.a;
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

template <class R, bool MHD>
struct StageSmem {
    static constexpr int NPV = MHD ? 10 : 6;
    static constexpr int NQ = MHD ? 10 : 5;
    static constexpr int NFI = (TI + 1) * TJ;
    static constexpr int NFJ = TI * (TJ + 1);
    static constexpr size_t bytes = sizeof(R) * (size_t)(4 * NPV * NT + NPV * NHALO + NQ * NFI + NQ * NFJ);
};

// STAGE 0: residual only (R_out = dUdt of U_in).  STAGE 1/2: predictor / corrector.
template <int STAGE, class R, bool MHD, int FLUX>
__global__ void __launch_bounds__(NT, MHD ? 1 : 2) stage_kernel(StageArgs A) {
    using SM = StageSmem<R, MHD>;
    constexpr int NPV = SM::NPV;
    constexpr int NQ = SM::NQ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* ring = reinterpret_cast<R*>(smem_raw);        // [4][NPV][NT]
    R* halo = ring + 4 * NPV * NT;                    // [NPV][NHALO]
    R* fI = halo + NPV * NHALO;                       // [NQ][NFI]
    R* fJ = fI + NQ * SM::NFI;                        // [NQ][NFJ]
    __shared__ double s_red[NT / 32];

    const Control* ctl = A.ctl;
    int parity = 0;
    double dt = 0.0, c_h = 0.0;
    if (STAGE != 0) {
        if (ctl->halted || ctl->status != ST_OK) return;
        if (STAGE == 2 && (ctl->n_fail > 0 || ctl->n_invalid1 > A.max_invalid_cells)) return;
        parity = ctl->step & 1;
        dt = ctl->dt_global;
    }
    c_h = ctl->c_h;
    const double* Uin = (STAGE == 0) ? A.U_in : A.Ubuf[parity];
    double* Uout = A.Ubuf[parity ^ 1];
    double damp = 1.0;
    if (MHD && A.P.divergence_cleaning && STAGE != 0) {
        // e4/fvcell.d:1068-1074 divergence_damping_factor
        double c_h2 = c_h * c_h;
        double c_p2 = 0.18 * A.P.divB_damping_length * c_h;
        damp = exp(-(c_h2 / c_p2) * dt);
    }

    const TileDesc t = A.tiles[blockIdx.x];
    const int blk = t.block;
    const BlockDesc& B = A.blocks[blk];
    const int ni_t = min(TI, B.n[0] - t.i0);
    const int nj_t = min(TJ, B.n[1] - t.j0);
    const int tid = threadIdx.x;
    const int ti = tid % TI, tj = tid / TI;
    const bool active = (ti < ni_t) && (tj < nj_t);
    const bool has_k = (A.P.dims == 3);
    const NumParams& P = A.P;

    // reconstruction weights of this block, shared by the CTA (kept out of registers)
    __shared__ R w[3][W_N];
    if (tid < 3 * W_N) w[tid / W_N][tid % W_N] = (R)B.w[tid / W_N][tid % W_N];
    const R c_hR = (R)c_h;

    // Prologue: interior states of planes k0-2 .. k0+1.
    const int kfirst = has_k ? t.k0 - 2 : t.k0;
    const int klast = has_k ? t.k0 + 2 : t.k0 + 1;
    if (active) {
        for (int kk = kfirst; kk < klast; ++kk) {
            Prim<double> s = load_cell<STAGE>(A, Uin, blk, t.i0 + ti, t.j0 + tj, kk, dt, damp);
            put_prim<R, NPV>(ring + (kk & 3) * NPV * NT, NT, tid, s);
        }
    }
    R fB[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) fB[q] = R(0);
    __syncthreads();
    if (active && has_k) {
        CellR<R> c[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) get_prim<R, NPV>(ring + ((t.k0 - 2 + m) & 3) * NPV * NT, NT, tid, c[m]);
        face_flux<R, MHD, FLUX, 2>(P, w[2], c_hR, c[0], c[1], c[2], c[3], fB);
    }
    __syncthreads();

    double sig_max = 0.0;
    const double Ai = B.area[0], Aj = B.area[1], Ak = B.area[2];
    const int nfi = (ni_t + 1) * nj_t;
    const int nfj = ni_t * (nj_t + 1);
    const int nh = 4 * nj_t + 4 * ni_t;

    for (int k = t.k0; k < t.k1; ++k) {
        // leading plane (k+2) interior and the halo of the current plane k
        if (active && has_k) {
            Prim<double> s = load_cell<STAGE>(A, Uin, blk, t.i0 + ti, t.j0 + tj, k + 2, dt, damp);
            put_prim<R, NPV>(ring + ((k + 2) & 3) * NPV * NT, NT, tid, s);
        }
        for (int h = tid; h < nh; h += NT) {
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
            Prim<double> s = load_cell<STAGE>(A, Uin, blk, t.i0 + hi, t.j0 + hj, k, dt, damp);
            put_prim<R, NPV>(halo, NHALO, h, s);
        }
        __syncthreads();

        const R* plane = ring + (k & 3) * NPV * NT;
        auto cell_at = [&](int ci, int cj, CellR<R>& c) {
            if (ci >= 0 && ci < ni_t && cj >= 0 && cj < nj_t) {
                get_prim<R, NPV>(plane, NT, ci + TI * cj, c);
            } else if (ci < 0 || ci >= ni_t) {
                int side = ci < 0 ? 0 : 1;
                int col = side == 0 ? ci + 2 : ci - ni_t;
                get_prim<R, NPV>(halo, NHALO, side * 2 * nj_t + col * nj_t + cj, c);
            } else {
                int side = cj < 0 ? 0 : 1;
                int row = side == 0 ? cj + 2 : cj - nj_t;
                get_prim<R, NPV>(halo, NHALO, 4 * nj_t + side * 2 * ni_t + row * ni_t + ci, c);
            }
        };

        R fT[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) fT[q] = R(0);
        if (active && has_k) {
            CellR<R> c[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) get_prim<R, NPV>(ring + ((k - 1 + m) & 3) * NPV * NT, NT, tid, c[m]);
            face_flux<R, MHD, FLUX, 2>(P, w[2], c_hR, c[0], c[1], c[2], c[3], fT);
        }
        for (int f = tid; f < nfi + nfj; f += NT) {
            CellR<R> c[4];
            R F[NQ];
            if (f < nfi) {
                int row = f / (ni_t + 1), fi = f % (ni_t + 1);
#pragma unroll
                for (int m = 0; m < 4; ++m) cell_at(fi - 2 + m, row, c[m]);
                face_flux<R, MHD, FLUX, 0>(P, w[0], c_hR, c[0], c[1], c[2], c[3], F);
                const int idx = fi + (TI + 1) * row;
#pragma unroll
                for (int q = 0; q < NQ; ++q) fI[q * SM::NFI + idx] = F[q];
            } else {
                int f2 = f - nfi;
                int fj = f2 / ni_t, col = f2 % ni_t;
#pragma unroll
                for (int m = 0; m < 4; ++m) cell_at(col, fj - 2 + m, c[m]);
                face_flux<R, MHD, FLUX, 1>(P, w[1], c_hR, c[0], c[1], c[2], c[3], F);
                const int idx = col + TI * fj;
#pragma unroll
                for (int q = 0; q < NQ; ++q) fJ[q * SM::NFJ + idx] = F[q];
            }
        }
        __syncthreads();

        if (active) {
            // e4/fvcell.d:824-856 time_derivatives: faces W, E, S, N, B, T
            const long long cell = cell_index(B, t.i0 + ti, t.j0 + tj, k);
            const long long g = B.offset + cell;
            double dU[NQ];
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                double FW = (double)fI[q * SM::NFI + ti + (TI + 1) * tj];
                double FE = (double)fI[q * SM::NFI + ti + 1 + (TI + 1) * tj];
                double FS = (double)fJ[q * SM::NFJ + ti + TI * tj];
                double FN = (double)fJ[q * SM::NFJ + ti + TI * (tj + 1)];
                double si = 0.0;
                si = __dsub_rn(si, d_mul(FW, -Ai));
                si = __dsub_rn(si, d_mul(FE, Ai));
                si = __dsub_rn(si, d_mul(FS, -Aj));
                si = __dsub_rn(si, d_mul(FN, Aj));
                if (has_k) {
                    si = __dsub_rn(si, d_mul((double)fB[q], -Ak));
                    si = __dsub_rn(si, d_mul((double)fT[q], Ak));
                }
                dU[q] = d_add(d_mul(B.vol_inv, si), 0.0);
            }
            if (STAGE == 0) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) A.R_out[(long long)q * A.total + g] = dU[q];
            } else {
                double U[10];
#pragma unroll
                for (int q = 0; q < NQ; ++q) U[q] = Uin[(long long)q * A.total + g];
                if (STAGE == 1) {
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        A.dU0[(long long)q * A.total + g] = dU[q];
                        U[q] = d_add(U[q], d_mul(dt, dU[q]));
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        double d0 = A.dU0[(long long)q * A.total + g];
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
                int st = decode(P, U, s, p, T);
                if (st != 0) {
                    atomicAdd(&A.ctl->n_fail, 1);
                    atomicMin(reinterpret_cast<unsigned long long*>(&A.ctl->first_bad_cell),
                              (unsigned long long)g);
                } else {
                    if (!check_data(P, s, p, T)) atomicAdd(STAGE == 1 ? &A.ctl->n_invalid1 : &A.ctl->n_invalid2, 1);
                    if (STAGE == 2) {
                        double sig = signal_frequency(P, B, s);
                        sig_max = fmax(sig_max, sig);
                        if (cell == (long long)B.n[0] * B.n[1] * B.n[2] - 1) A.last_signal[blk] = sig;
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) fB[q] = fT[q];
        __syncthreads();
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
}

}  // namespace gdfv
