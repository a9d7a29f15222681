// Host-side views of a context shared between the translation units of libgdfv.so.
#pragma once
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "gdfv_device.cuh"

namespace gdfv {

// What the allocation-free step (gdfv_noalloc.cu) needs of a context.
struct NoallocView {
    int prepared, precision, flux, mhd, nblocks, max_invalid_cells;
    long long total;
    int nq, n_tiles, n_tiles2;   // n_tiles2 > 0: the corrector's table follows the first
    const BlockDesc* d_blocks;
    const TileDesc* d_tiles;
    const InflowState* d_inflow;
    const double* d_rot;         // exchange rotations (9 doubles each), null if none
    NumParams P;
    double c_h;
    cudaStream_t stream;
    int persistent;
    long long max_block_cells;   // cells of the largest block
};
bool noalloc_view(int ctx, NoallocView* v);
void noalloc_set_error(int ctx, const std::string& msg);
// Records the failing cell (global index g) for gdfv_last_bad_cell and returns its
// description for an error message ("" when g names no cell).
std::string noalloc_bad_cell_text(int ctx, long long g);

// What the adjoint (gdfv_adjoint.cu) needs of a context (gdfv_runtime.cu).
struct AdjView {
    int prepared, flux, mhd, precision, nblocks, ninflow, dims;
    long long total;
    const BlockDesc* d_blocks;
    const InflowState* d_inflow;
    const double* d_rot;    // exchange rotations (9 doubles each), null if none
    NumParams P;
    double c_h;             // the GLM wave speed the context holds (MHD residual)
    cudaStream_t stream;
    std::vector<BlockDesc> h_blocks;
    double** scratch;       // context-owned, lazily allocated adjoint buffers
    long long* scratch_n;
    int* scratch_ready;     // 1 once the face offsets in the scratch are uploaded
};
bool adjoint_view(int ctx, AdjView* v);
void adjoint_set_error(int ctx, const std::string& msg);

// Fixed-dt step chains (gdfv_runtime.cu), for the adjoint's recomputation.
int steps_dt_prepare(int ctx);
cudaError_t enqueue_steps_dt(int ctx, cudaStream_t stream, const double* U_in, double* const* U_out,
                             double* const* U1_out, const double* dts, int n, bool fresh);
int steps_dt_status(int ctx, cudaStream_t stream);
cudaError_t enqueue_step_ch(int ctx, cudaStream_t stream, const double* U, double dt, double* out);
cudaStream_t context_aux_stream(int ctx, int which);

}  // namespace gdfv
