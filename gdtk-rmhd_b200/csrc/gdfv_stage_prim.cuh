// gdfv_stage_prim.cuh -- the Euler stage kernel of the default options (van Albada
// limiter and extrema clipping on, e4 epsilon, no outflow boundary with a flux or ghost
// rule of its own, uniform blocks, 3D), in both flux precisions R: float (the FP32-flux /
// FP64-update form) and double (the plain FP64 form, bit for bit the reference's
// arithmetic as stage_kernel's FP64 path).  Same stage semantics and the same per-face
// arithmetic as stage_kernel (recon_cell, face_flux; the stage update, the decode
// checks and the signal reduction in FP64), with a leaner data flow:
//
// * Decoded primitives in HBM.  Every stage decodes the state it produces in its
//   update phase anyway (the checks of decode_conserved, e4/fvcell.d:586-822); it also
//   stores that state's primitives (rho, vel, u, a) in R, SoA [6][total]: the predictor
//   those of U1 = U0 + dt dU0, the corrector those of U2.  The next stage loads its
//   stencils -- own column, halo and prologue planes -- from these six values instead of
//   loading and decoding ten FP64 values (U0 and dU0) per stencil cell.  In FP64 the
//   stored primitives are the bits the stencil decode would give (decode and
//   decode_prim perform the same operations).  P[b] holds the primitives of state
//   buffer b; P1 those of the predictor state.
// * i direction in registers.  Warp w of the tile owns row w, lane l cell l.  The
//   reconstruction of the lane's own cell gives both its interface values; the left
//   state of face l-1/2 comes from lane l-1 by a warp shuffle, the flux of face
//   l+1/2 likewise, so neither the reconstructed states nor the fluxes of the i faces
//   pass through shared memory.  The j direction passes the plus-side state and the
//   flux of each row's south face to the next row through shared memory.
// * Edge warp.  The tile edges -- reconstruction of the cells beyond the last column
//   and row on each side, the east faces of the rows and the north faces of the top
//   row -- go to one extra warp, whose lanes take one edge item each, instead of one
//   lane of each row warp (a divergent lane costs the whole warp's issue slots).
//
// Per plane k (ring of four planes k .. k+3 in shared memory, padded by the 2-cell halo):
//   A  issue the loads of the lead plane k+3 (own columns) and of the halo of plane k+1
//   B  rows: i and j reconstruction of plane k; edge warp: edge reconstructions;
//      then the loads of A into the ring (their latency hides behind B)       | barrier
//   C  rows: W, S faces, then k reconstruction and T face; edge: E, N faces   | barrier
//   D  rows: residual (faces W, E, S, N, B, T), update, decode, checks, P of the result
// Two barriers per plane: A and B of plane k+1 touch only ring slots and exchange
// arrays that nothing reads between the barrier after C of plane k and the barrier
// after B of plane k+1.
// Only the states that must cross a barrier are kept in registers across it (the i
// and j minus-side states, the W and T face fluxes, the k plus-side state and the B
// face flux carried from plane to plane); the S face flux is read back from shared
// memory, where the row above needs it anyway.
#pragma once
#include "gdfv_stage.cuh"

namespace gdfv {

// Primitives of one cell as the ring stores them (rho, v0, v1, v2, u, a).
template <class R>
struct PF {
    R rho, v[3], u, a;
};

template <class R>
__device__ __forceinline__ PF<R> load_pf(const R* __restrict__ Pin, long long total, long long g) {
    PF<R> c;
    c.rho = __ldg(Pin + g);
    c.v[0] = __ldg(Pin + total + g);
    c.v[1] = __ldg(Pin + 2 * total + g);
    c.v[2] = __ldg(Pin + 3 * total + g);
    c.u = __ldg(Pin + 4 * total + g);
    c.a = __ldg(Pin + 5 * total + g);
    return c;
}

template <class R>
__device__ __forceinline__ void put_pf(R* base, int stride, int idx, const PF<R>& c) {
    base[idx] = c.rho;
    base[stride + idx] = c.v[0];
    base[2 * stride + idx] = c.v[1];
    base[3 * stride + idx] = c.v[2];
    base[4 * stride + idx] = c.u;
    base[5 * stride + idx] = c.a;
}

// A cell that lies outside the block (at most one index outside): the ghost that
// the boundary condition of that face synthesises (resolve() names the source), from
// the float primitives of its source cells.  The rules of stage_kernel's ghost
// synthesis: mirror with negated normal velocity (internal_copy_then_reflect.d),
// copy or linear extrapolation of rho, u and velocity with a from the boundary cell
// (extrapolate_copy.d:124-201), the fixed inflow state (flow_state_copy.d), or the
// partner block's cell (full_face_copy.d; exchanges with an Rmatrix run stage_kernel).
template <class R>
__device__ __forceinline__ PF<R> ghost_pf(const StageArgs& A, const R* __restrict__ Pin, const BlockDesc& B, int i, int j,
                                       int k) {
    const CellSrc s = resolve<false, false>(A, B, i, j, k);
    PF<R> c;
    if (s.kind == SRC_INFLOW) {
        const InflowState& in = A.inflow[s.inflow];
        c.rho = (R)in.rho; c.u = (R)in.u; c.a = (R)in.a;
        c.v[0] = (R)in.vel[0]; c.v[1] = (R)in.vel[1]; c.v[2] = (R)in.vel[2];
        return c;
    }
    c = load_pf(Pin, A.total, s.blk->offset + s.c0);
    if (s.kind == SRC_MIRROR) {
        c.v[s.axis] = -c.v[s.axis];
    } else if (s.kind == SRC_EXTRAP1_G0 || s.kind == SRC_EXTRAP1_G1) {
        // g0 = 2 e - f1, g1 = 2 g0 - e (e the boundary cell, f1 the cell inside it)
        const PF<R> f1 = load_pf(Pin, A.total, s.blk->offset + s.c1);
        PF<R> g = c;
        g.rho = R(2) * c.rho - f1.rho;
        g.u = R(2) * c.u - f1.u;
        for (int m = 0; m < 3; ++m) g.v[m] = R(2) * c.v[m] - f1.v[m];
        if (s.kind == SRC_EXTRAP1_G1) {
            PF<R> h = c;
            h.rho = R(2) * g.rho - c.rho;
            h.u = R(2) * g.u - c.u;
            for (int m = 0; m < 3; ++m) h.v[m] = R(2) * g.v[m] - c.v[m];
            return h;
        }
        return g;
    }
    return c;
}

// Asynchronous copy of one cell's six primitives from P into a padded ring plane
// (cp.async: global to shared memory without passing through registers; the copies of
// a thread complete at cp_async_wait).
template <class R>
__device__ __forceinline__ void cp_async_pf(R* base, int stride, int idx, const R* Pin, long long total, long long g) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(base + q * stride + idx);
        if constexpr (sizeof(R) == 4)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(Pin + q * total + g) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(Pin + q * total + g) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's committed copy groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Primitives of a decoded FP64 state (what the next stage loads).
template <class R>
__device__ __forceinline__ void store_pf(R* __restrict__ Pout, long long total, long long g, const Prim<double>& s) {
    Pout[g] = (R)s.rho;
    Pout[total + g] = (R)s.v[0];
    Pout[2 * total + g] = (R)s.v[1];
    Pout[3 * total + g] = (R)s.v[2];
    Pout[4 * total + g] = (R)s.u;
    Pout[5 * total + g] = (R)s.a;
}

// Shared-memory layout (values of R) of the kernel for TJ row warps and tiles TW cells
// wide: TW = 32, one row per warp; TW = 16, two rows per warp (lanes 0-15 and 16-31),
// NR = TJ * 32 / TW rows.
template <class R, int TJ_, int TW = 32>
struct GeoF {
    static_assert(TW == 32 || TW == 16, "tiles 32 or 16 cells wide");
    static constexpr int TI = TW, TJ = TJ_, NR = TJ_ * (32 / TW);
    static constexpr int NT = 32 * (TJ + 1);
    static constexpr int PW = TI + 4, PH = NR + 4, PLANE = PW * PH;
    static constexpr int NS = 5;                              // reconstructed scalars
    static constexpr int O_RING = 0;                          // [4][6][PLANE]
    static constexpr int O_QPJ = O_RING + 4 * 6 * PLANE;      // [NS][NR][TI]   j plus-side state of each cell
    static constexpr int O_EJS = O_QPJ + NS * NR * TI;        // [NS][TI]       j plus-side state of row -1
    static constexpr int O_EJN = O_EJS + NS * TI;             // [NS][TI]       j minus-side state of row nj
    static constexpr int O_EIW = O_EJN + NS * TI;             // [NS][NR]       i plus-side state of column -1
    static constexpr int O_EIE = O_EIW + NS * NR;             // [NS][NR]       i minus-side state of column ni
    static constexpr int O_EIL = O_EIE + NS * NR;             // [NS][NR]       i plus-side state of column ni-1
    static constexpr int O_FJ = O_EIL + NS * NR;              // [NS][NR+1][TI] flux of the S face of rows 0..nj
    static constexpr int O_FIE = O_FJ + NS * (NR + 1) * TI;   // [NS][NR]       flux of the E face of each row
    static constexpr int O_END = O_FIE + NS * NR;
    static constexpr size_t bytes = sizeof(R) * (size_t)O_END;
};

// Resident CTAs per SM each precision's kernel is compiled for (its register budget).
#ifndef GDFV_MINB_PRIM_FP32
#define GDFV_MINB_PRIM_FP32 3
#endif
#ifndef GDFV_MINB_PRIM_FP64
#define GDFV_MINB_PRIM_FP64 2
#endif

template <class R, int STAGE, int FLUX, int TJ, int PERS, int TW = 32>
__global__ void __launch_bounds__(32 * (TJ + 1), sizeof(R) == 4 ? GDFV_MINB_PRIM_FP32 : GDFV_MINB_PRIM_FP64)
    stage_prim_kernel(StageArgs A) {
    static_assert(STAGE == 1 || STAGE == 2, "predictor or corrector");
    constexpr bool FAST = sizeof(R) == 4;
    using G = GeoF<R, TJ, TW>;
    constexpr int TI = G::TI, NR = G::NR, PW = G::PW, PLANE = G::PLANE, NS = G::NS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* sm = reinterpret_cast<R*>(smem_raw);
    R* ring = sm + G::O_RING;
    R* QPJ = sm + G::O_QPJ;
    R* EJS = sm + G::O_EJS;
    R* EJN = sm + G::O_EJN;
    R* EIW = sm + G::O_EIW;
    R* EIE = sm + G::O_EIE;
    R* EIL = sm + G::O_EIL;
    R* FJ = sm + G::O_FJ;
    R* FIE = sm + G::O_FIE;
    __shared__ double s_red[TJ + 1];
    __shared__ R w[3][W_N];
    __shared__ R wf[3][WF_N];
    __shared__ int s_tile;
    __shared__ double s_geo[4];   // 1/dx, 1/dy, 1/dz, 1/volume of the tile's block

    const Control* ctl = A.ctl;
    if (ctl->halted || ctl->status != ST_OK) return;
    if (STAGE == 2 && (ctl->n_fail > 0 || ctl->n_invalid1 > A.max_invalid_cells)) return;
    const int parity = ctl->step & 1;
    const double dt = ctl->dt_global;
    const double* __restrict__ Uin = A.Ubuf[parity];
    double* Uout = A.Ubuf[parity ^ 1];
    const R* __restrict__ Pin = static_cast<const R*>(STAGE == 1 ? A.prim[parity] : A.prim1);
    R* Pout = static_cast<R*>(STAGE == 1 ? A.prim1 : A.prim[parity ^ 1]);
    const long long total = A.total;
    const NumParams& P = A.P;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool edge = warp == TJ;   // the edge warp
    // own column and row in the tile: lane and warp (32 wide), or two rows per warp (16 wide)
    const int ti = TW == 32 ? lane : (lane & (TW - 1));
    const int tj = TW == 32 ? warp : warp * (32 / TW) + lane / TW;

    Control* qctl = const_cast<Control*>(ctl);
    int tix = blockIdx.x;
    if (PERS) {
        if (tid == 0) s_tile = (int)atomicAdd(&qctl->tile_next, 1u);
        __syncthreads();
        tix = s_tile;
    }
    while (tix < A.n_tiles) {
        const TileDesc t = A.tiles[tix];
        const int blk = t.block;
        const BlockDesc& B = A.blocks[blk];
        const int ni_t = min(TI, B.n[0] - t.i0);
        const int nj_t = min(NR, B.n[1] - t.j0);
        const bool active = !edge && tj < nj_t && ti < ni_t;
        const int pidx = (ti + 2) + PW * (tj + 2);         // own cell in a padded plane
        if (tid < 3 * W_N) w[tid / W_N][tid % W_N] = (R)B.w[tid / W_N][tid % W_N];
        if (tid < 3) {
            s_geo[tid] = 1.0 / B.len[tid];
            const double* bw = B.w[tid];
            const double tc = bw[W_TOC];
            wf[tid][WF_EPS] = (R)(P.eps_van_albada / (tc * tc));
            wf[tid][WF_P1] = (R)(bw[W_AL0] * tc * bw[W_TWOL]);
            wf[tid][WF_P2] = (R)(bw[W_AL0] * tc * bw[W_LENL0]);
            wf[tid][WF_R1] = (R)(bw[W_AR0] * tc * bw[W_LENL0]);
            wf[tid][WF_R2] = (R)(bw[W_AR0] * tc * bw[W_TWOL]);
        }
        if (tid == 3) s_geo[3] = B.vol_inv;
        __syncthreads();

        const int n2 = B.n[2];
        const int pstride = B.n[0] * B.n[1];
        const long long boff = B.offset;
        int c_own = (t.i0 + ti) + B.n[0] * ((t.j0 + tj) + B.n[1] * t.k0);
        auto slot = [&](int kk) -> R* { return ring + (kk & 3) * (6 * PLANE); };

        double sig_max = 0.0;
        // halo cell of this thread in every plane: 2 columns beside each row, 2 rows
        // above and below the tile; the edge warp takes items 0..31, the row threads the rest
        const int nh = 4 * nj_t + 4 * ni_t;
        const int h = edge ? lane : tid + 32;
        const bool h_on = h < nh;
        int h_ci = 0, h_cj = 0, h_dst = 0;
        if (h_on) {
            int hi, hj;
            if (h < 4 * nj_t) {
                const int side = h / (2 * nj_t), rem = h % (2 * nj_t);
                const int col = rem / nj_t, row = rem % nj_t;
                hi = side == 0 ? col - 2 : ni_t + col;
                hj = row;
            } else {
                const int h2 = h - 4 * nj_t;
                const int side = h2 / (2 * ni_t), rem = h2 % (2 * ni_t);
                const int row = rem / ni_t, col = rem % ni_t;
                hj = side == 0 ? row - 2 : nj_t + row;
                hi = col;
            }
            h_ci = t.i0 + hi;
            h_cj = t.j0 + hj;
            h_dst = (hi + 2) + PW * (hj + 2);
        }
        const bool h_in = h_on && h_ci >= 0 && h_ci < B.n[0] && h_cj >= 0 && h_cj < B.n[1];
        // in-block index of the halo cell in plane k0 (advanced one plane per step)
        int c_halo = (h_in ? h_ci : 0) + B.n[0] * ((h_in ? h_cj : 0) + B.n[1] * t.k0);
        // edge items of phases B and C (edge warp): reconstruction of 2 nj + 2 ni cells,
        // fluxes of nj east faces and ni north faces
        const int ne_rec = 2 * nj_t + 2 * ni_t, ne_flux = nj_t + ni_t;
        R kq_prev_p[NS];   // k plus-side state of the current plane (left state of its top face)
        R fB[NS];          // flux through the bottom face of the own cell
        // ---------------- prologue: planes k0-2 .. k0+2 of the own column, halo of plane k0
        if (h_in) {
            put_pf(slot(t.k0), PLANE, h_dst, load_pf(Pin, total, boff + c_halo));
        } else if (h_on) {
            put_pf(slot(t.k0), PLANE, h_dst, ghost_pf(A, Pin, B, h_ci, h_cj, t.k0));
        }
        c_halo += pstride;
        if (active) {
            const int gi = t.i0 + ti, gj = t.j0 + tj;
            PF<R> c[5];
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const int kk = t.k0 - 2 + m;
                c[m] = (kk >= 0 && kk < n2) ? load_pf(Pin, total, boff + (c_own + (m - 2) * pstride))
                                            : ghost_pf(A, Pin, B, gi, gj, kk);
            }
            put_pf(slot(t.k0 - 1), PLANE, pidx, c[1]);
            put_pf(slot(t.k0), PLANE, pidx, c[2]);
            put_pf(slot(t.k0 + 1), PLANE, pidx, c[3]);
            put_pf(slot(t.k0 + 2), PLANE, pidx, c[4]);
            R qm1[NS], q0[NS], qp1[NS], qm[NS], qpkm1[NS];
            // face-local order for k: v2, v0, v1, rho, u
            auto fr = [](const PF<R>& x, R* q) { q[0] = x.v[2]; q[1] = x.v[0]; q[2] = x.v[1]; q[3] = x.rho; q[4] = x.u; };
            fr(c[0], qm1); fr(c[1], q0); fr(c[2], qp1);
            recon_cell<R, NS, false, 1>(w[2], wf[2], P, qm1, q0, qp1, qm, qpkm1);
            fr(c[1], qm1); fr(c[2], q0); fr(c[3], qp1);
            recon_cell<R, NS, false, 1>(w[2], wf[2], P, qm1, q0, qp1, qm, kq_prev_p);
            face_flux<R, false, FLUX, 2, 6>(P, R(0), qpkm1, qm, slot(t.k0 - 1), pidx, slot(t.k0), pidx, PLANE, fB);
        }


        __syncthreads();

        for (int k = t.k0; k < t.k1; ++k) {
            R* cur = slot(k);
            R* nx1 = slot(k + 1);
            R* nx2 = slot(k + 2);
            // ---------------- A: copies of the lead plane k+3 (own columns) and the halo of plane
            // k+1 into the ring, in flight during B (slot k+3 held plane k-1, last read in C of
            // plane k-1; the halo positions of slot k+1 are read first in B of plane k+1)
            // (only while a plane k+1 follows in this tile: then k+3 <= n2+1, a ghost at most one
            // layer deep, and k+1 < n2 lies inside the block)
            const bool more = k + 1 < t.k1;
            const bool lead_in = active && more && k + 3 < n2;
            if (lead_in) cp_async_pf(slot(k + 3), PLANE, pidx, Pin, total, boff + (c_own + 3 * pstride));
            if (h_in && more) cp_async_pf(nx1, PLANE, h_dst, Pin, total, boff + c_halo);
            cp_async_commit();

            // ---------------- B: i and j reconstruction
            R qLi[NS], qmi[NS], qmj[NS];
            {
                R qpi[NS];
                if (active) {
                    R qm1[NS], q0[NS], qp1[NS], qpj[NS];
                    gather<R, NS, 0>(cur, PLANE, pidx - 1, qm1);
                    gather<R, NS, 0>(cur, PLANE, pidx, q0);
                    gather<R, NS, 0>(cur, PLANE, pidx + 1, qp1);
                    recon_cell<R, NS, false, 1>(w[0], wf[0], P, qm1, q0, qp1, qmi, qpi);
                    if (ti == ni_t - 1) {
#pragma unroll
                        for (int s = 0; s < NS; ++s) EIL[s * NR + tj] = qpi[s];
                    }
                    gather<R, NS, 1>(cur, PLANE, pidx - PW, qm1);
                    gather<R, NS, 1>(cur, PLANE, pidx, q0);
                    gather<R, NS, 1>(cur, PLANE, pidx + PW, qp1);
                    recon_cell<R, NS, false, 1>(w[1], wf[1], P, qm1, q0, qp1, qmj, qpj);
#pragma unroll
                    for (int s = 0; s < NS; ++s) QPJ[(s * NR + tj) * TI + ti] = qpj[s];
                } else {
#pragma unroll
                    for (int s = 0; s < NS; ++s) qpi[s] = R(0);
                }
                // left state of the W face: the plus-side state of the lane to the left
#pragma unroll
                for (int s = 0; s < NS; ++s) qLi[s] = __shfl_up_sync(0xffffffffu, qpi[s], 1, TI);
            }
            if (edge) {
                for (int e = lane; e < ne_rec; e += 32) {
                    R qm1[NS], q0[NS], qp1[NS], qm[NS], qp[NS];
                    if (e < 2 * nj_t) {            // column -1 (plus side) or ni (minus side) of row r
                        const bool east = e >= nj_t;
                        const int r = east ? e - nj_t : e;
                        const int p = (east ? ni_t + 2 : 1) + PW * (r + 2);
                        gather<R, NS, 0>(cur, PLANE, p - 1, qm1);
                        gather<R, NS, 0>(cur, PLANE, p, q0);
                        gather<R, NS, 0>(cur, PLANE, p + 1, qp1);
                        recon_cell<R, NS, false, 1>(w[0], wf[0], P, qm1, q0, qp1, qm, qp);
                        R* dst = east ? EIE : EIW;
#pragma unroll
                        for (int s = 0; s < NS; ++s) dst[s * NR + r] = east ? qm[s] : qp[s];
                    } else {                       // row -1 (plus side) or nj (minus side) of column c
                        const int e2 = e - 2 * nj_t;
                        const bool north = e2 >= ni_t;
                        const int c = north ? e2 - ni_t : e2;
                        const int p = (c + 2) + PW * (north ? nj_t + 2 : 1);
                        gather<R, NS, 1>(cur, PLANE, p - PW, qm1);
                        gather<R, NS, 1>(cur, PLANE, p, q0);
                        gather<R, NS, 1>(cur, PLANE, p + PW, qp1);
                        recon_cell<R, NS, false, 1>(w[1], wf[1], P, qm1, q0, qp1, qm, qp);
                        R* dst = north ? EJN : EJS;
#pragma unroll
                        for (int s = 0; s < NS; ++s) dst[s * TI + c] = north ? qm[s] : qp[s];
                    }
                }
            }
            // ghosts of A (boundary tiles), then the copies complete
            if (active && more && !lead_in)
                put_pf(slot(k + 3), PLANE, pidx, ghost_pf(A, Pin, B, t.i0 + ti, t.j0 + tj, k + 3));
            if (h_on && more && !h_in) put_pf(nx1, PLANE, h_dst, ghost_pf(A, Pin, B, h_ci, h_cj, k + 1));
            cp_async_wait<0>();
            __syncthreads();

            // ---------------- C: fluxes (W, S faces; k reconstruction and the T face)
            R fW[NS], fT[NS];
            if (active) {
                if (ti == 0) {
#pragma unroll
                    for (int s = 0; s < NS; ++s) qLi[s] = EIW[s * NR + tj];
                }
                face_flux<R, false, FLUX, 0, 6>(P, R(0), qLi, qmi, cur, pidx - 1, cur, pidx, PLANE, fW);
                {
                    R qL[NS], fS[NS];
#pragma unroll
                    for (int s = 0; s < NS; ++s)
                        qL[s] = tj == 0 ? EJS[s * TI + ti] : QPJ[(s * NR + tj - 1) * TI + ti];
                    face_flux<R, false, FLUX, 1, 6>(P, R(0), qL, qmj, cur, pidx - PW, cur, pidx, PLANE, fS);
#pragma unroll
                    for (int s = 0; s < NS; ++s) FJ[(s * (NR + 1) + tj) * TI + ti] = fS[s];
                }
                {
                    R qm1[NS], q0[NS], qp1[NS], kq_m[NS], kq_p[NS];
                    gather<R, NS, 2>(cur, PLANE, pidx, qm1);
                    gather<R, NS, 2>(nx1, PLANE, pidx, q0);
                    gather<R, NS, 2>(nx2, PLANE, pidx, qp1);
                    recon_cell<R, NS, false, 1>(w[2], wf[2], P, qm1, q0, qp1, kq_m, kq_p);
                    face_flux<R, false, FLUX, 2, 6>(P, R(0), kq_prev_p, kq_m, cur, pidx, nx1, pidx, PLANE, fT);
#pragma unroll
                    for (int s = 0; s < NS; ++s) kq_prev_p[s] = kq_p[s];
                }
            } else {
#pragma unroll
                for (int s = 0; s < NS; ++s) fW[s] = R(0);
            }
            if (edge) {
                for (int e = lane; e < ne_flux; e += 32) {
                    R qL[NS], qR[NS], F[NS];
                    if (e < nj_t) {                // E face of row e
                        const int p = (ni_t + 2) + PW * (e + 2);
#pragma unroll
                        for (int s = 0; s < NS; ++s) { qL[s] = EIL[s * NR + e]; qR[s] = EIE[s * NR + e]; }
                        face_flux<R, false, FLUX, 0, 6>(P, R(0), qL, qR, cur, p - 1, cur, p, PLANE, F);
#pragma unroll
                        for (int s = 0; s < NS; ++s) FIE[s * NR + e] = F[s];
                    } else {                       // N face of the top row, column c
                        const int c = e - nj_t;
                        const int p = (c + 2) + PW * (nj_t + 2);
#pragma unroll
                        for (int s = 0; s < NS; ++s) {
                            qL[s] = QPJ[(s * NR + nj_t - 1) * TI + c];
                            qR[s] = EJN[s * TI + c];
                        }
                        face_flux<R, false, FLUX, 1, 6>(P, R(0), qL, qR, cur, p - PW, cur, p, PLANE, F);
#pragma unroll
                        for (int s = 0; s < NS; ++s) FJ[(s * (NR + 1) + nj_t) * TI + c] = F[s];
                    }
                }
            }
            __syncthreads();

            // ---------------- D: residual (e4/fvcell.d:824-856, faces W, E, S, N, B, T) and update
            {
                // flux of the E face: the W face of the lane to the right
                R fE[NS];
#pragma unroll
                for (int s = 0; s < NS; ++s) fE[s] = __shfl_down_sync(0xffffffffu, fW[s], 1, TI);
                if (active) {
                    if (ti == ni_t - 1) {
#pragma unroll
                        for (int s = 0; s < NS; ++s) fE[s] = FIE[s * NR + tj];
                    }
                    // face_flux turned the face-local flux (mass, normal and tangential momentum,
                    // energy) back to the global frame: F[MASS], F[XMOM..ZMOM], F[TOTENERGY]
                    const long long g = boff + c_own;
                    const double Vi = s_geo[3];
                    const double Ai = B.area[0], Aj = B.area[1], Ak = B.area[2];
                    double dU[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) {
                        const R fS = FJ[(q * (NR + 1) + tj) * TI + ti];
                        const R fN = FJ[(q * (NR + 1) + tj + 1) * TI + ti];
                        if constexpr (FAST) {
                            // float: differences of opposite faces in float (same-signed, nearly
                            // equal fluxes subtract exactly), the sum in FP64
                            const R dI = fW[q] - fE[q];
                            const R dJ = fS - fN;
                            double si = (double)dI * Ai + (double)dJ * Aj;
                            si += (double)(fB[q] - fT[q]) * Ak;
                            dU[q] = Vi * si;
                        } else {
                            // FP64: the reference's sum over the faces in their order, without
                            // contraction (time_derivatives, e4/fvcell.d:824-856)
                            double si = 0.0;
                            si = __dsub_rn(si, d_mul(fW[q], -Ai));
                            si = __dsub_rn(si, d_mul(fE[q], Ai));
                            si = __dsub_rn(si, d_mul(fS, -Aj));
                            si = __dsub_rn(si, d_mul(fN, Aj));
                            si = __dsub_rn(si, d_mul(fB[q], -Ak));
                            si = __dsub_rn(si, d_mul(fT[q], Ak));
                            dU[q] = d_add(d_mul(Vi, si), 0.0);
                        }
                    }
                    double U[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) U[q] = __ldg(Uin + (long long)q * total + g);
                    if (STAGE == 1) {
#pragma unroll
                        for (int q = 0; q < 5; ++q) {
                            A.dU0[(long long)q * total + g] = dU[q];
                            U[q] = d_add(U[q], d_mul(dt, dU[q]));
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < 5; ++q) {
                            const double d0 = __ldg(A.dU0 + (long long)q * total + g);
                            U[q] = d_add(U[q], d_mul(dt, d_add(d_mul(0.5, d0), d_mul(0.5, dU[q]))));
                            Uout[(long long)q * total + g] = U[q];
                        }
                    }
                    Prim<double> s;
                    double p, T;
                    const int st = FAST ? decode_fast(P, U, s, p, T) : decode(P, U, s, p, T);
                    if (st != 0) {
                        atomicAdd(&A.ctl->n_fail, 1);
                        atomicMin(reinterpret_cast<unsigned long long*>(&A.ctl->first_bad_cell),
                                  (unsigned long long)g);
                    } else {
                        store_pf(Pout, total, g, s);
                        if (!check_data(P, s, p, T)) {
                            atomicAdd(STAGE == 1 ? &A.ctl->n_invalid1 : &A.ctl->n_invalid2, 1);
                            atomicMin(reinterpret_cast<unsigned long long*>(&A.ctl->first_bad_cell),
                                      (unsigned long long)g);
                        }
                        if (STAGE == 2) {
                            const double inv_len[3] = {s_geo[0], s_geo[1], s_geo[2]};
                            const double sig = FAST ? signal_fast(P, inv_len, s) : signal_frequency(P, B.len, s);
                            sig_max = fmax(sig_max, sig);
                            if (c_own == pstride * n2 - 1) A.last_signal[blk] = sig;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < NS; ++q) fB[q] = fT[q];
                }
            }
            c_own += pstride;
            c_halo += pstride;
        }

        if (STAGE == 2) {
            // CTA max of the signal frequency -> one atomic per CTA (dt rule input)
            for (int o = 16; o > 0; o >>= 1) sig_max = fmax(sig_max, __shfl_xor_sync(0xffffffffu, sig_max, o));
            if (lane == 0) s_red[warp] = sig_max;
            __syncthreads();
            if (tid == 0) {
                double m = s_red[0];
                for (int wv = 1; wv <= TJ; ++wv) m = fmax(m, s_red[wv]);
                atomicMax(&A.max_signal[blk], (unsigned long long)__double_as_longlong(m));
            }
        }
        if (!PERS) break;
        __syncthreads();
        if (tid == 0) s_tile = (int)atomicAdd(&qctl->tile_next, 1u);
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

// Primitives of the state U (decode_prim; for float, with the float-flux reciprocal and
// square root), for P[b] of a state set from outside a stage.
template <class R>
__global__ void prims_kernel(const double* __restrict__ U, long long total, NumParams P, R* __restrict__ Pout) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= total) return;
    double u[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) u[q] = U[q * total + g];
    Prim<double> s;
    decode_prim<sizeof(R) == 4, false>(P, u, s);
    store_pf(Pout, total, g, s);
}

}  // namespace gdfv
