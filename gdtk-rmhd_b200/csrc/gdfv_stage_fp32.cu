// gdfv_stage_fp32.cu -- instantiations of the fused stage kernel with float flux
// arithmetic.  The conserved state, the residual sums and the RK update stay
// in FP64 in both variants.
#include "gdfv_launch.h"
#define GDFV_REAL float
#define GDFV_TJ TJ_FP32
#define GDFV_TJ_CORR TJ_FP32_CORR
#define GDFV_TJ_MHD TJ_FP32_MHD
#define GDFV_TJ_MHD_CORR TJ_FP32_MHD_CORR
#define GDFV_LAUNCH launch_stage_fp32
#define GDFV_CONFIGURE configure_stage_fp32
#define GDFV_PRIM_PATH 1
#define GDFV_PRIMS prims_fp32
#include "gdfv_stage_inst.cuh"
