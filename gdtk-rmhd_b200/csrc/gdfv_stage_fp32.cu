// gdfv_stage_fp32.cu -- instantiations of the fused stage kernel with float flux
// arithmetic.  The conserved state, the residual sums and the RK update stay
// in FP64 in both variants.
#include "gdfv_launch.h"

namespace gdfv {

namespace {
using Real = float;
constexpr int TJ = TJ_FP32;

template <int STAGE, bool MHD, int FLUX>
cudaError_t launch_one(const StageArgs& A, cudaStream_t s) {
    using G = Geo<Real, MHD, TJ>;
    // defaults (limiter and extrema clipping on) take the specialised path
    if (A.P.apply_limiter && A.P.extrema_clipping)
        stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1><<<A.n_tiles, G::NT, G::bytes, s>>>(A);
    else
        stage_kernel<STAGE, Real, MHD, FLUX, TJ, 0><<<A.n_tiles, G::NT, G::bytes, s>>>(A);
    return cudaGetLastError();
}

template <int STAGE, bool MHD, int FLUX>
cudaError_t configure_one() {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<STAGE, Real, MHD, FLUX, TJ, 0>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)Geo<Real, MHD, TJ>::bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(stage_kernel<STAGE, Real, MHD, FLUX, TJ, 1>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Geo<Real, MHD, TJ>::bytes);
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
cudaError_t configure_t() {
    cudaError_t e;
    if ((e = configure_one<STAGE, true, FLUX_HLLE>()) != cudaSuccess) return e;
    if ((e = configure_one<STAGE, false, FLUX_AUSMDV>()) != cudaSuccess) return e;
    return configure_one<STAGE, false, FLUX_HLLC>();
}
}  // namespace

cudaError_t launch_stage_fp32(int stage, int flux, bool mhd, const StageArgs& A, cudaStream_t s) {
    if (A.n_tiles <= 0) return cudaSuccess;
    switch (stage) {
    case 0: return launch_stage_t<0>(flux, mhd, A, s);
    case 1: return launch_stage_t<1>(flux, mhd, A, s);
    case 2: return launch_stage_t<2>(flux, mhd, A, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t configure_stage_fp32() {
    cudaError_t e;
    if ((e = configure_t<0>()) != cudaSuccess) return e;
    if ((e = configure_t<1>()) != cudaSuccess) return e;
    return configure_t<2>();
}

}  // namespace gdfv
