// gdfv_launch.h -- interface between the host runtime and the two kernel
// translation units (FP64 flux and FP32 flux, compiled with different flags).
#pragma once
#include <cuda_runtime.h>

#include "gdfv_stage.cuh"

namespace gdfv {

// Rows of cells per column tile (the tile is 32 x TJ columns) of each flux precision.
#ifndef GDFV_TJ_FP64
#define GDFV_TJ_FP64 6
#endif
#ifndef GDFV_TJ_FP32
#define GDFV_TJ_FP32 8
#endif
// rows of the float-flux MHD kernels (their ten variables need more shared memory per row)
#ifndef GDFV_TJ_FP32_MHD
#define GDFV_TJ_FP32_MHD 7
#endif
// rows of the float-flux Euler corrector: with 7 rows its CTAs of 256 threads get 80
// registers (fewer spills) at the same 3 CTAs per SM
#ifndef GDFV_TJ_FP32_CORR
#define GDFV_TJ_FP32_CORR 7
#endif
// rows of the FP64 MHD kernels (one CTA per SM: their shared memory allows no second)
#ifndef GDFV_TJ_FP64_MHD
#define GDFV_TJ_FP64_MHD 7
#endif
// rows of the FP64 Euler corrector (by default those of the FP64 kernels)
#ifndef GDFV_TJ_FP64_CORR
#define GDFV_TJ_FP64_CORR GDFV_TJ_FP64
#endif
// rows of the float-flux MHD corrector (by default those of the float MHD kernels)
#ifndef GDFV_TJ_FP32_MHD_CORR
#define GDFV_TJ_FP32_MHD_CORR GDFV_TJ_FP32_MHD
#endif
constexpr int TJ_FP64 = GDFV_TJ_FP64;
constexpr int TJ_FP32_MHD_CORR = GDFV_TJ_FP32_MHD_CORR;
constexpr int TJ_FP64_CORR = GDFV_TJ_FP64_CORR;
constexpr int TJ_FP64_MHD = GDFV_TJ_FP64_MHD;
constexpr int TJ_FP32_CORR = GDFV_TJ_FP32_CORR;
constexpr int TJ_FP32 = GDFV_TJ_FP32;
constexpr int TJ_FP32_MHD = GDFV_TJ_FP32_MHD;

// Rows per column tile of the kernels a run launches.
inline int tile_rows(int precision, bool mhd) {
    return precision == 0 ? (mhd ? TJ_FP64_MHD : TJ_FP64) : (mhd ? TJ_FP32_MHD : TJ_FP32);
}
// Rows per column tile of the corrector (stage 2) of a run.
inline int tile_rows_corrector(int precision, bool mhd) {
    return precision == 0 ? (mhd ? TJ_FP64_MHD : TJ_FP64_CORR) : (mhd ? TJ_FP32_MHD_CORR : TJ_FP32_CORR);
}

// Options under which the float-flux Euler stages run the kernel on decoded primitives
// (gdfv_stage_prim.cuh) when the arguments carry primitive buffers (the FP64 form keeps
// stage_kernel, which ran faster than an FP64 build of the primitive kernel): the
// defaults (limiter and extrema clipping on, e4 epsilon), no outflow boundary with a
// flux or ghost rule of its own, no graded block, no exchange with an Rmatrix, 3D.
inline bool prim_path(const NumParams& P) {
    return !P.mhd && P.apply_limiter && P.extrema_clipping && !P.lmr_epsilon && !P.outflow_bcs && !P.graded &&
           !P.rotating && P.dims == 3;
}

// Launch one stage (0 = residual only, 1 = predictor, 2 = corrector) over A.n_tiles tiles.
cudaError_t launch_stage_fp64(int stage, int flux, bool mhd, const StageArgs& A, cudaStream_t s);
cudaError_t launch_stage_fp32(int stage, int flux, bool mhd, const StageArgs& A, cudaStream_t s);
// Primitives (rho, vel, u, a; SoA [6][total], float or double) of the state U, for the
// kernels on decoded primitives, enqueued on stream s.
void prims_fp32(const double* U, long long total, const NumParams& P, void* Pout, cudaStream_t s);
// Raise the dynamic shared-memory limit of every instantiation (once per device).
cudaError_t configure_stage_fp64();
cudaError_t configure_stage_fp32();

}  // namespace gdfv
