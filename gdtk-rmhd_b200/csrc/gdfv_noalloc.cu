// gdfv_noalloc.cu -- one predictor-corrector step on caller-owned device arrays
// that allocates no device memory.
//
// Some callers cannot call cudaMalloc: an application that gives all device
// memory to its own pool allocator (a framework's caching allocator, for
// example) and forbids other allocations, or a real-time loop that cannot
// accept cudaMalloc's latency and implicit device synchronisation.  For them,
// gdfv_step_noalloc takes the step's scratch memory (the predictor derivative,
// the step-control record and the per-block signal maxima) from one file-scope
// device array, reserved when the library is loaded on a device and kept until
// the process exits.
//
// Limits and sharing:
//   * the derivative needs nq * (cells of all blocks) doubles; calls that need
//     more than GDFV_NOALLOC_MAX_VALUES are rejected with GDFV_ERR_ARG;
//     at most GDFV_NOALLOC_MAX_BLOCKS blocks;
//   * every call on a device uses the same array, so calls whose kernels
//     overlap on the GPU (two host threads, or two streams) race on it; calls
//     issued one after another on one stream are safe: each call clears the
//     counters and signal maxima it needs before its kernels run;
//   * the first call on a device resolves the array's device address
//     (cudaGetSymbolAddress) and caches it, so make that first call before any
//     stream capture begins on that device.  A cached address that no longer
//     names device memory (the device was reset, cudaDeviceReset, and its
//     context made anew) is looked up again;
//   * MHD with divergence cleaning: c_h is the rule of a gdfv_run step
//     (e4/simcore.d:1625-1648 update_ch_for_divergence_cleaning with
//     e4/fluidblock.d:975-995) applied to the signal frequency of U_in, which a
//     first kernel reduces per block into the scratch.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>
#include <string>

#include "../../include/gdfv.h"
#include "gdfv_internal.h"
#include "gdfv_launch.h"

namespace gdfv {

namespace {

constexpr long long kMaxValues = GDFV_NOALLOC_MAX_VALUES;
constexpr int kMaxBlocks = GDFV_NOALLOC_MAX_BLOCKS;
// layout in doubles: [derivative | control record | signal maxima | last-cell signals]
constexpr long long kCtlOffset = kMaxValues;
constexpr long long kCtlDoubles = ((sizeof(Control) + 255) / 256) * 32;
constexpr long long kSigOffset = kCtlOffset + kCtlDoubles;
constexpr long long kLastOffset = kSigOffset + kMaxBlocks;
constexpr long long kTotalDoubles = kLastOffset + kMaxBlocks;

// The scratch.  In host code this name is only a host-side stand-in for the
// device symbol: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_step_scratch[kTotalDoubles];

std::mutex g_mu;
double* g_addr[64] = {nullptr};

// Resets the step-control record and the signal maxima of this call.
__global__ void noalloc_begin_kernel(Control* c, unsigned long long* maxsig, int nblocks, double dt, double c_h) {
    if (blockIdx.x != 0) return;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) maxsig[b] = 0ull;
    if (threadIdx.x == 0) {
        c->time = 0.0; c->dt_global = dt; c->c_h = c_h; c->cfl_max = 0.0; c->dt_allow = 0.0;
        c->max_time = 0.0; c->t0 = 0.0; c->first_bad_cell = LLONG_MAX;
        c->step = 0; c->step_limit = 1; c->status = ST_OK; c->halted = 0;
        c->n_fail = 0; c->n_invalid1 = 0; c->n_invalid2 = 0;
        c->attempt = 0; c->retrying = 0; c->steps_done = 0;
        c->tile_next = 0; c->tile_done = 0;
    }
}

// Per-block maximum of the signal frequency of U (e4/fvcell.d:975-1059) into
// maxsig[blockIdx.y] (bit patterns of positive doubles), as the initial scan of a
// gdfv_run does.
__global__ void noalloc_signal_kernel(const double* U, long long total, const BlockDesc* blocks, NumParams P,
                                      unsigned long long* maxsig) {
    const int blk = blockIdx.y;
    const BlockDesc& B = blocks[blk];
    const long long n = (long long)B.n[0] * B.n[1] * B.n[2];
    double sig = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        double u[10];
        for (int q = 0; q < P.nq; ++q) u[q] = U[q * total + B.offset + c];
        Prim<double> s;
        double p, T;
        if (decode(P, u, s, p, T) == 0) {
            double L[3];
            cell_lengths(B, (int)(c % B.n[0]), (int)((c / B.n[0]) % B.n[1]), (int)(c / ((long long)B.n[0] * B.n[1])), L);
            sig = fmax(sig, signal_frequency(P, L, s));
        }
    }
    for (int o = 16; o > 0; o >>= 1) sig = fmax(sig, __shfl_xor_sync(0xffffffffu, sig, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&maxsig[blk], (unsigned long long)__double_as_longlong(sig));
}

// c_h from the signal maxima with the operations of the step controller's rule
// (cfl_max = signal dt, c_h = min over blocks of cfl_max L_min / dt); then the
// maxima are cleared for the corrector's reduction.
__global__ void noalloc_ch_kernel(Control* c, const BlockDesc* blocks, unsigned long long* maxsig, int nblocks) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = c->dt_global;
    for (int b = 0; b < nblocks; ++b) {
        const double smax = __longlong_as_double((long long)maxsig[b]);
        const double cfl_max = smax * dt;
        const double ch = cfl_max * blocks[b].L_min / dt;
        c->c_h = b == 0 ? ch : fmin(ch, c->c_h);
        maxsig[b] = 0ull;
    }
}

}  // namespace
}  // namespace gdfv

using namespace gdfv;

extern "C" int gdfv_step_noalloc(int ctx, const double* U_in_dev, double* U_out_dev, double dt, int* n_bad_cells) {
    NoallocView v;
    if (!noalloc_view(ctx, &v)) return GDFV_ERR_ARG;
    if (!v.prepared) { noalloc_set_error(ctx, "call gdfv_prepare first"); return GDFV_ERR_STATE; }
    if (!U_in_dev || !U_out_dev || U_in_dev == U_out_dev || !(dt > 0.0)) {
        noalloc_set_error(ctx, "gdfv_step_noalloc needs distinct input/output arrays and dt > 0");
        return GDFV_ERR_ARG;
    }
    if ((long long)v.nq * v.total > kMaxValues || v.nblocks > kMaxBlocks) {
        noalloc_set_error(ctx, "gdfv_step_noalloc: problem exceeds the fixed scratch (nq*cells > " +
                                   std::to_string(kMaxValues) + " values or more than " +
                                   std::to_string(kMaxBlocks) + " blocks)");
        return GDFV_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        noalloc_set_error(ctx, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return GDFV_ERR_CUDA;
    }
    double* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_addr[dev]) {
            // a device reset ends the context the cached address belonged to
            cudaPointerAttributes at{};
            if (cudaPointerGetAttributes(&at, g_addr[dev]) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
                cudaGetLastError();
                g_addr[dev] = nullptr;
            }
        }
        if (!g_addr[dev]) {
            // once per device, with that device current
            e = cudaGetSymbolAddress((void**)&g_addr[dev], g_step_scratch);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                noalloc_set_error(ctx, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return GDFV_ERR_CUDA;
            }
        }
        base = g_addr[dev];
    }
    Control* ctl = reinterpret_cast<Control*>(base + kCtlOffset);
    unsigned long long* maxsig = reinterpret_cast<unsigned long long*>(base + kSigOffset);
    double* lastsig = base + kLastOffset;

    StageArgs A{};
    A.blocks = v.d_blocks;
    A.tiles = v.d_tiles;
    A.inflow = v.d_inflow;
    A.rot = v.d_rot;
    A.Ubuf[0] = const_cast<double*>(U_in_dev);  // read by both stages (step parity 0)
    A.Ubuf[1] = U_out_dev;                      // written by the corrector
    A.dU0 = base;
    A.ctl = ctl;
    A.max_signal = maxsig;
    A.last_signal = lastsig;
    A.total = v.total;
    A.P = v.P;
    A.n_tiles = v.n_tiles;
    A.n_tiles2 = v.n_tiles2;
    A.max_invalid_cells = v.max_invalid_cells;
    A.persistent = v.persistent;

    noalloc_begin_kernel<<<1, 256, 0, v.stream>>>(ctl, maxsig, v.nblocks, dt, 0.0);
    e = cudaGetLastError();
    if (e == cudaSuccess && v.mhd && v.P.divergence_cleaning) {
        const long long per = (v.max_block_cells + 255) / 256;
        const dim3 grid((unsigned)(per < 256 ? per : 256), (unsigned)v.nblocks);
        noalloc_signal_kernel<<<grid, 256, 0, v.stream>>>(U_in_dev, v.total, v.d_blocks, v.P, maxsig);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            noalloc_ch_kernel<<<1, 32, 0, v.stream>>>(ctl, v.d_blocks, maxsig, v.nblocks);
            e = cudaGetLastError();
        }
    }
    for (int stage = 1; stage <= 2 && e == cudaSuccess; ++stage) {
        e = v.precision == 0 ? launch_stage_fp64(stage, v.flux, v.mhd, A, v.stream)
                             : launch_stage_fp32(stage, v.flux, v.mhd, A, v.stream);
    }
    Control h{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, ctl, sizeof(Control), cudaMemcpyDeviceToHost, v.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) {
        noalloc_set_error(ctx, std::string("gdfv_step_noalloc: ") + cudaGetErrorString(e));
        return GDFV_ERR_CUDA;
    }
    if (n_bad_cells) *n_bad_cells = h.n_fail + h.n_invalid1 + h.n_invalid2;
    if (h.n_fail > 0) {
        noalloc_set_error(ctx, "gdfv_step_noalloc: a cell failed to decode; U_out is not a valid step." +
                                   noalloc_bad_cell_text(ctx, h.first_bad_cell));
        return GDFV_ERR_STEP_FAILED;
    }
    if (h.n_invalid1 > v.max_invalid_cells || h.n_invalid2 > v.max_invalid_cells) {
        noalloc_set_error(ctx, "gdfv_step_noalloc: too many bad cells." + noalloc_bad_cell_text(ctx, h.first_bad_cell));
        return GDFV_ERR_BAD_CELLS;
    }
    return GDFV_OK;
}
