// gdfv_stage_inst.cuh -- launch and configuration of the stage-kernel
// instantiations of one flux precision.  Included once by each precision's
// translation unit, which defines GDFV_REAL, GDFV_TJ (Euler rows), GDFV_TJ_CORR (Euler
// corrector rows), GDFV_TJ_MHD, GDFV_TJ_MHD_CORR, GDFV_LAUNCH and
// GDFV_CONFIGURE first.
#include "gdfv_launch.h"
#if GDFV_PRIM_PATH
#include "gdfv_stage_prim.cuh"
#endif

namespace gdfv {

namespace {
using Real = GDFV_REAL;
constexpr int TJ_E = GDFV_TJ;        // Euler kernels
constexpr int TJ_E2 = GDFV_TJ_CORR;  // Euler corrector (stage 2)
constexpr int TJ_M = GDFV_TJ_MHD;    // MHD kernels
constexpr int TJ_M2 = GDFV_TJ_MHD_CORR;  // MHD corrector (stage 2)

// Rows of the kernels of a stage: a corrector may have a second instantiation with
// its own rows (TJ_E2, TJ_M2), launched over the corrector's tile table when the
// runtime built one (n_tiles2 > 0).
template <bool MHD>
constexpr int rows() { return MHD ? TJ_M : TJ_E; }
template <bool MHD>
constexpr int rows_corrector() { return MHD ? TJ_M2 : TJ_E2; }

template <class K>
cudaError_t set_smem(K k, size_t bytes) {
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Resident CTAs on the device (CTAs per SM x SMs) of the persistent
// instantiation: the grid of the persistent launch.
template <int STAGE, bool MHD, int FLUX, int TJ>
int& resident() {
    static int v = 0;
    return v;
}

template <int STAGE, bool MHD, int FLUX, int TJ>
cudaError_t launch_rows(const StageArgs& A, cudaStream_t s) {
    using G = Geo<Real, MHD, TJ>;
    // defaults (limiter and extrema clipping on, e4 epsilon, none of the outflow
    // boundaries with their own ghost or flux rule, uniform blocks, no exchange with an
    // Rmatrix) take the specialised path, which also has the persistent form
    if (A.P.apply_limiter && A.P.extrema_clipping && !A.P.lmr_epsilon && !A.P.outflow_bcs && !A.P.graded &&
        !A.P.rotating) {
        const int cap = resident<STAGE, MHD, FLUX, TJ>();
        if (A.persistent && cap > 0)
            stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1, 1><<<cap < A.n_tiles ? cap : A.n_tiles, G::NT, G::bytes, s>>>(A);
        else
            stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1, 0><<<A.n_tiles, G::NT, G::bytes, s>>>(A);
    } else {
        stage_kernel<STAGE, Real, MHD, FLUX, TJ, 0, 0><<<A.n_tiles, G::NT, G::bytes, s>>>(A);
    }
    return cudaGetLastError();
}

#if GDFV_PRIM_PATH
// The Euler kernel on decoded primitives (gdfv_stage_prim.cuh): TJ_E row warps, tiles 32
// or 16 cells wide (TW).
template <int STAGE, int FLUX, int TW>
int& resident_prim() {
    static int v = 0;
    return v;
}

template <int STAGE, int FLUX, int TW>
cudaError_t launch_prim_w(const StageArgs& A, cudaStream_t s) {
    using G = GeoF<Real, TJ_E, TW>;
    const int cap = resident_prim<STAGE, FLUX, TW>();
    if (A.persistent && cap > 0)
        stage_prim_kernel<Real, STAGE, FLUX, TJ_E, 1, TW><<<cap < A.n_tiles ? cap : A.n_tiles, G::NT, G::bytes, s>>>(A);
    else
        stage_prim_kernel<Real, STAGE, FLUX, TJ_E, 0, TW><<<A.n_tiles, G::NT, G::bytes, s>>>(A);
    return cudaGetLastError();
}

// Over the first tile table (rows TJ_E in both stages), or over its own tables: tiles 32
// wide, then (a second launch; a persistent launch leaves the tile queue at zero) tiles
// 16 wide.  The runtime fills one of the two.
template <int STAGE, int FLUX>
cudaError_t launch_prim(const StageArgs& A, cudaStream_t s) {
    if (A.n_prim_wide + A.n_prim_narrow == 0) return launch_prim_w<STAGE, FLUX, 32>(A, s);
    cudaError_t e = cudaSuccess;
    StageArgs Ap = A;
    Ap.tiles = A.tiles + A.n_tiles + A.n_tiles2;
    if (A.n_prim_wide > 0) {
        Ap.n_tiles = A.n_prim_wide;
        e = launch_prim_w<STAGE, FLUX, 32>(Ap, s);
        Ap.tiles += A.n_prim_wide;
    }
    if (e == cudaSuccess && A.n_prim_narrow > 0) {
        Ap.n_tiles = A.n_prim_narrow;
        e = launch_prim_w<STAGE, FLUX, 16>(Ap, s);
    }
    return e;
}

template <int STAGE, int FLUX, int TW>
cudaError_t configure_prim_w(int n_sm) {
    using G = GeoF<Real, TJ_E, TW>;
    cudaError_t e = set_smem(stage_prim_kernel<Real, STAGE, FLUX, TJ_E, 0, TW>, G::bytes);
    if (e == cudaSuccess) e = set_smem(stage_prim_kernel<Real, STAGE, FLUX, TJ_E, 1, TW>, G::bytes);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_prim_kernel<Real, STAGE, FLUX, TJ_E, 1, TW>,
                                                      G::NT, G::bytes);
    if (e != cudaSuccess) return e;
    resident_prim<STAGE, FLUX, TW>() = per_sm * n_sm;
    return cudaSuccess;
}

template <int STAGE, int FLUX>
cudaError_t configure_prim(int n_sm) {
    cudaError_t e = configure_prim_w<STAGE, FLUX, 32>(n_sm);
    return e == cudaSuccess ? configure_prim_w<STAGE, FLUX, 16>(n_sm) : e;
}
#endif

template <int STAGE, bool MHD, int FLUX>
cudaError_t launch_one(const StageArgs& A, cudaStream_t s) {
#if GDFV_PRIM_PATH
    if constexpr (!MHD && STAGE >= 1) {
        if (A.prim[0] && prim_path(A.P)) return launch_prim<STAGE, FLUX>(A, s);
    }
#endif
    if constexpr (STAGE == 2 && rows_corrector<MHD>() != rows<MHD>()) {
        if (A.n_tiles2 > 0) {   // the corrector's own tile table follows the first
            StageArgs A2 = A;
            A2.tiles = A.tiles + A.n_tiles;
            A2.n_tiles = A.n_tiles2;
            return launch_rows<2, MHD, FLUX, rows_corrector<MHD>()>(A2, s);
        }
    }
    return launch_rows<STAGE, MHD, FLUX, rows<MHD>()>(A, s);
}

template <int STAGE, bool MHD, int FLUX, int TJ>
cudaError_t configure_rows(int n_sm) {
    using G = Geo<Real, MHD, TJ>;
    cudaError_t e = set_smem(stage_kernel<STAGE, Real, MHD, FLUX, TJ, 0, 0>, G::bytes);
    if (e == cudaSuccess) e = set_smem(stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1, 0>, G::bytes);
    if (e == cudaSuccess) e = set_smem(stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1, 1>, G::bytes);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1, 1>, G::NT,
                                                      G::bytes);
    if (e != cudaSuccess) return e;
    resident<STAGE, MHD, FLUX, TJ>() = per_sm * n_sm;
    return cudaSuccess;
}

template <int STAGE, bool MHD, int FLUX>
cudaError_t configure_one(int n_sm) {
    cudaError_t e = configure_rows<STAGE, MHD, FLUX, rows<MHD>()>(n_sm);
#if GDFV_PRIM_PATH
    if constexpr (!MHD && STAGE >= 1)
        if (e == cudaSuccess) e = configure_prim<STAGE, FLUX>(n_sm);
#endif
    if constexpr (STAGE == 2 && rows_corrector<MHD>() != rows<MHD>())
        if (e == cudaSuccess) e = configure_rows<2, MHD, FLUX, rows_corrector<MHD>()>(n_sm);
    return e;
}

template <int STAGE>
cudaError_t launch_stage_t(int flux, bool mhd, const StageArgs& A, cudaStream_t s) {
    if (mhd) {
        if (flux == FLUX_HLLE) return launch_one<STAGE, true, FLUX_HLLE>(A, s);
        return cudaErrorInvalidValue;
    }
    if (flux == FLUX_AUSMDV) return launch_one<STAGE, false, FLUX_AUSMDV>(A, s);
    if (flux == FLUX_HLLC) return launch_one<STAGE, false, FLUX_HLLC>(A, s);
    return cudaErrorInvalidValue;
}

template <int STAGE>
cudaError_t configure_t(int n_sm) {
    cudaError_t e;
    if ((e = configure_one<STAGE, true, FLUX_HLLE>(n_sm)) != cudaSuccess) return e;
    if ((e = configure_one<STAGE, false, FLUX_AUSMDV>(n_sm)) != cudaSuccess) return e;
    return configure_one<STAGE, false, FLUX_HLLC>(n_sm);
}
}  // namespace

cudaError_t GDFV_LAUNCH(int stage, int flux, bool mhd, const StageArgs& A, cudaStream_t s) {
    if (A.n_tiles <= 0) return cudaSuccess;
    switch (stage) {
    case 0: return launch_stage_t<0>(flux, mhd, A, s);
    case 1: return launch_stage_t<1>(flux, mhd, A, s);
    case 2: return launch_stage_t<2>(flux, mhd, A, s);
    }
    return cudaErrorInvalidValue;
}

#if GDFV_PRIM_PATH
void GDFV_PRIMS(const double* U, long long total, const NumParams& P, void* Pout, cudaStream_t s) {
    prims_kernel<Real><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(U, total, P, static_cast<Real*>(Pout));
}
#endif

cudaError_t GDFV_CONFIGURE() {
    int dev = 0, n_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if ((e = configure_t<0>(n_sm)) != cudaSuccess) return e;
    if ((e = configure_t<1>(n_sm)) != cudaSuccess) return e;
    return configure_t<2>(n_sm);
}

}  // namespace gdfv
