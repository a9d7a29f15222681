// gdfv_stage_fp64.cu -- instantiations of the fused stage kernel with double flux
// arithmetic (compiled without FMA contraction: bit-reproducible against the
// CPU restatement).
#include "gdfv_launch.h"
#define GDFV_REAL double
#define GDFV_TJ TJ_FP64
#define GDFV_TJ_CORR TJ_FP64_CORR
#define GDFV_TJ_MHD TJ_FP64_MHD
#define GDFV_TJ_MHD_CORR TJ_FP64_MHD
#define GDFV_LAUNCH launch_stage_fp64
#define GDFV_CONFIGURE configure_stage_fp64
#include "gdfv_stage_inst.cuh"
