// gdfv_runtime.cu -- host runtime behind the C ABI (include/gdfv.h): contexts,
// configuration by the reference's option names, block and boundary tables,
// device memory, the device-resident step controller and CUDA-graph replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gdfv.h"
#include "gdfv_internal.h"
#include "gdfv_launch.h"

namespace gdfv {

// ---------------------------------------------------------------- device kernels
struct StepParams {
    int cfl_count, n_stages, fixed_time_step, mhd_cleaning;
    int max_attempts, max_invalid_cells, nblocks, pad_;
    double cfl_value, dt_init, dt_max;
};

// e4/simcore_gasdynamic_step.d:60-160 (global dt rule) with the block rule of
// e4/fluidblock.d:998-1095 and c_h of e4/fluidblock.d:975-995 / e4/simcore.d:1625-1648.
// One thread; inputs are the per-block maxima of the signal frequency that the
// previous corrector stage (or the initial scan) left behind.
__global__ void step_begin_kernel(Control* c, const BlockDesc* blocks, unsigned long long* maxsig,
                                  const double* lastsig, StepParams sp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (c->halted || c->status != ST_OK) return;
    if (c->step >= c->step_limit || (c->max_time > 0.0 && c->time >= c->max_time)) {
        c->halted = 1;
        return;
    }
    if (!c->retrying) {
        if (!sp.fixed_time_step && (c->step % sp.cfl_count) == 0) {
            const double cfl_allow = sp.n_stages == 1 ? 0.9 : (sp.n_stages == 2 ? 1.2 : 1.6);
            const double cfl_adjust = 0.5;
            const bool check_cfl = c->step > 0;
            double dt_allow_all = 1.79769313486231570e+308;
            double cfl_max_all = 0.0;
            for (int b = 0; b < sp.nblocks; ++b) {
                double smax = __longlong_as_double((long long)maxsig[b]);
                // max over cells of (dt*signal) and min of (cfl/signal) follow from the max signal
                double cfl_max = c->dt_global * smax;
                double dt_allow = sp.cfl_value / smax;
                if (check_cfl && (cfl_max < 0.0 || cfl_max > cfl_allow)) {
                    cfl_max = cfl_adjust * cfl_allow;
                    dt_allow = cfl_max / lastsig[b];  // signal of the last cell visited
                }
                dt_allow_all = fmin(dt_allow_all, dt_allow);
                cfl_max_all = fmax(cfl_max_all, cfl_max);
            }
            c->dt_allow = dt_allow_all;
            c->cfl_max = cfl_max_all;
            if (c->step == 0) c->dt_allow = fmin(sp.dt_init, c->dt_allow);
            if (c->dt_allow <= c->dt_global) {
                c->dt_global = c->dt_allow;
            } else {
                c->dt_global = fmin(c->dt_global * 1.5, c->dt_allow);
                c->dt_global = fmin(c->dt_global, sp.dt_max);
            }
        }
        if (sp.mhd_cleaning) {
            bool first = true;
            for (int b = 0; b < sp.nblocks; ++b) {
                double smax = __longlong_as_double((long long)maxsig[b]);
                double cfl_max = smax * c->dt_global;
                double ch = cfl_max * blocks[b].L_min / c->dt_global;
                c->c_h = first ? ch : fmin(ch, c->c_h);
                first = false;
            }
        }
        c->t0 = c->time;
    }
    c->n_fail = 0;
    c->n_invalid1 = 0;
    c->n_invalid2 = 0;
    c->first_bad_cell = LLONG_MAX;
    for (int b = 0; b < sp.nblocks; ++b) maxsig[b] = 0ull;
}

// Phase 14 and the retry loop of e4/simcore_gasdynamic_step.d:1437-1560.
__global__ void step_end_kernel(Control* c, StepParams sp) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (c->halted || c->status != ST_OK) return;
    if (c->n_fail > 0) {
        c->attempt += 1;
        c->dt_global = c->dt_global * 0.2;
        if (c->attempt >= sp.max_attempts) {
            c->status = ST_DECODE_FAILED;
            c->halted = 1;
        } else {
            c->retrying = 1;
        }
        return;
    }
    if (c->n_invalid1 > sp.max_invalid_cells || c->n_invalid2 > sp.max_invalid_cells) {
        c->status = ST_TOO_MANY_BAD_CELLS;
        c->halted = 1;
        return;
    }
    c->time = c->t0 + c->dt_global;
    c->step += 1;
    c->attempt = 0;
    c->retrying = 0;
    c->steps_done += 1;
}

struct BlockRange {
    long long offset, n;
    int blk;
};

// rhoT -> conserved (update_thermo_from_rhoT then encode_conserved)
__global__ void encode_rhoT_kernel(const double* prim, long long n, double* U, long long total, long long offset,
                                   NumParams P, int* bad) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= n) return;
    double rho = prim[c], vx = prim[n + c], vy = prim[2 * n + c], vz = prim[3 * n + c], T = prim[4 * n + c];
    double Bx = prim[5 * n + c], By = prim[6 * n + c], Bz = prim[7 * n + c], psi = prim[8 * n + c];
    if (T <= 0.0 || rho <= 0.0) { atomicAdd(bad, 1); return; }
    double u = P.gas.Cv * T;
    const long long g = offset + c;
    U[MASS * total + g] = rho;
    U[XMOM * total + g] = rho * vx;
    U[YMOM * total + g] = rho * vy;
    U[ZMOM * total + g] = rho * vz;
    double ke = 0.5 * (vx * vx + vy * vy + vz * vz);
    double E = rho * (u + ke);
    if (P.mhd) {
        U[XB * total + g] = Bx; U[YB * total + g] = By; U[ZB * total + g] = Bz;
        U[PSI * total + g] = psi; U[DIVB * total + g] = 0.0;
        double me = 0.5 * (Bx * Bx + By * By + Bz * Bz);
        E = E + me;
    }
    U[TOTENERGY * total + g] = E;
}

__global__ void decode_kernel(const double* U, long long total, long long offset, long long n, NumParams P,
                              double* out) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= n) return;
    double u[10];
    for (int q = 0; q < P.nq; ++q) u[q] = U[q * total + offset + c];
    Prim<double> s;
    double p = 0, T = 0;
    int st = decode(P, u, s, p, T);
    if (st != 0) { s.a = p = T = nan(""); }
    double v[12] = {s.rho, s.v[0], s.v[1], s.v[2], s.u, p, T, s.a, s.B[0], s.B[1], s.B[2], s.psi};
    for (int q = 0; q < 12; ++q) out[q * n + c] = v[q];
}

// Signal frequency of the current state: per-block max and the last cell's value.
__global__ void signal_scan_kernel(const double* U, long long total, const BlockDesc* blocks, int blk, NumParams P,
                                   unsigned long long* maxsig, double* lastsig, int* bad) {
    const BlockDesc& B = blocks[blk];
    long long n = (long long)B.n[0] * B.n[1] * B.n[2];
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double sig = 0.0;
    if (c < n) {
        double u[10];
        for (int q = 0; q < P.nq; ++q) u[q] = U[q * total + B.offset + c];
        Prim<double> s;
        double p, T;
        if (decode(P, u, s, p, T) == 0) {
            double L[3];
            cell_lengths(B, (int)(c % B.n[0]), (int)((c / B.n[0]) % B.n[1]), (int)(c / ((long long)B.n[0] * B.n[1])), L);
            sig = signal_frequency(P, L, s);
            if (c == n - 1) lastsig[blk] = sig;
        } else {
            atomicAdd(bad, 1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) sig = fmax(sig, __shfl_xor_sync(0xffffffffu, sig, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&maxsig[blk], (unsigned long long)__double_as_longlong(sig));
}

// ---------------------------------------------------------------- host side
struct HostBC {
    int type = BC_SLIP_WALL;
    int x_order = 0;
    int other = -1, other_face = -1;
    int orientation = 0;      // exchange: ExchangeBC_FullFace orientation 0..3
    int rotate = 0;           // exchange: rot holds an Rmatrix for the ghosts' vectors
    double rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double inflow[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
};

struct HostBlock {
    int n[3];
    double len[3];
    double origin[3];
    HostBC bc[6];
    long long offset = 0;
    std::vector<double> vert[3];   // graded: vertex coordinates along each axis (n + 1 each)
    bool graded() const { return !vert[0].empty(); }
    double cell_len(int d, int c) const { return graded() ? vert[d][c + 1] - vert[d][c] : len[d]; }
};

struct Config {
    int flux = FLUX_AUSMDV;
    int precision = 0;  // 0 fp64, 1 fp32 flux
    int dims = 3;
    int mhd = 0, divergence_cleaning = 0;
    int apply_limiter = 1, extrema_clipping = 1, apply_entropy_fix = 1, glm_reference_indexing = 1;
    int stringent_cfl = 0, cfl_count = 10, max_attempts = 3, max_invalid_cells = 0;
    int fixed_time_step = 0;
    int tile_kchunk = 0;  // 0: chosen per block
    int tile_width = 32;  // kernel on decoded primitives: tiles 32 or 16 cells wide (build_tiles)
    int persistent = 0;   // 1: stage kernels as a resident grid taking tiles from a queue
    int autotune = 0;     // time tile shapes and the launch form on the first run, keep the fastest
    int lmr_epsilon = 0;  // van_albada_variant = lmr
    double cfl_value = 0.5, dt_init = 1.0e-3, dt_max = 1.0e-3;
    double eps_van_albada = 1.0e-12, R = 287.1, gamma = 1.4, divB_damping_length = 1.0;
    double max_velocity = 30000.0, max_temp = 50000.0, min_temp = 0.0;
};

struct Context {
    Config cfg;
    std::vector<HostBlock> blocks;
    bool prepared = false;
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    long long total = 0;
    int nq = 5;
    int n_tiles = 0;
    int n_tiles2 = 0;   // > 0: the corrector's tile table (other rows) follows the first in d_tiles
    int n_prim_wide = 0, n_prim_narrow = 0;   // the primitive kernel's tables after those
    double* U[2] = {nullptr, nullptr};
    double* dU0 = nullptr;
    BlockDesc* d_blocks = nullptr;
    TileDesc* d_tiles = nullptr;
    InflowState* d_inflow = nullptr;
    Control* d_ctl = nullptr;
    Control* h_ctl = nullptr;  // pinned mirror
    unsigned long long* d_maxsig = nullptr;
    double* d_lastsig = nullptr;
    int* d_bad = nullptr;
    std::vector<BlockDesc> h_blocks;
    NumParams P{};
    StepParams sp{};
    cudaGraphExec_t graph = nullptr;    // kGraphSteps step slots
    cudaGraphExec_t graph1 = nullptr;   // one step slot (the tail of a run)
    int graph_steps = 0;
    bool signal_valid = false;
    int n_inflow = 0;
    size_t tiles_cap = 0;              // capacity of d_tiles (entries)
    bool tuned = false;
    double tune_ms = 0.0;              // stage-1 + stage-2 time of the tuned configuration
    double* adj_scratch = nullptr;     // adjoint work arrays, allocated on first use
    double* jvp_scratch = nullptr;     // Frechet JVP work arrays (U + sigma v, R0, R1, partial sums)
    double* norm_scratch = nullptr;    // per-CTA partials and result of gdfv_residual_norms
    double* d_geom = nullptr;          // graded blocks: cell lengths and l2r2 weights per direction
    double* d_rot = nullptr;           // rotations of exchange faces with an Rmatrix, 9 doubles each
    double* d_rec = nullptr;           // gdfv_run_record: dt of each step, then a flag
    int rec_cap = 0;
    int adj_ready = 0;
    long long adj_scratch_n = 0;
    cudaStream_t aux_stream[2] = {nullptr, nullptr};  // lowest / highest priority streams of the rollout adjoint
    void* prim[2] = {nullptr, nullptr};   // primitives of U[0], U[1] (kernels on decoded primitives)
    void* prim1 = nullptr;             // primitives of the predictor state
    bool prims_valid = false;          // prim[parity] holds the primitives of the current state
    long long last_bad_cell = -1;      // global index of the cell the last failure reported (-1: none)
    std::vector<double> h_inflow;      // supersonic-inflow states as uploaded, 9 doubles each (p, T, vel, B, psi)
    Control* step_ctl = nullptr;       // control record of gdfv_step_dt
    unsigned long long* step_maxsig = nullptr;
    double* step_lastsig = nullptr;
    unsigned long long* ch_maxsig = nullptr;   // signal scan of the MHD step adjoint (its own stream)
    double* ch_lastsig = nullptr;
    int* ch_bad = nullptr;   // cells the c_h scans could not decode: counted, never read (the
                             // stages' own decode checks report a failed step)

    ~Context() {
        if (graph) cudaGraphExecDestroy(graph);
        if (graph1) cudaGraphExecDestroy(graph1);
        for (void* p : {(void*)U[0], (void*)U[1], (void*)dU0, (void*)d_blocks, (void*)d_tiles, (void*)d_inflow,
                        (void*)d_ctl, (void*)d_maxsig, (void*)d_lastsig, (void*)d_bad, (void*)adj_scratch, (void*)jvp_scratch,
                        (void*)norm_scratch, (void*)prim[0], (void*)prim[1], (void*)prim1, (void*)d_geom, (void*)d_rot, (void*)d_rec,
                        (void*)step_ctl, (void*)step_maxsig, (void*)step_lastsig, (void*)ch_maxsig,
                        (void*)ch_lastsig, (void*)ch_bad})
            if (p) cudaFree(p);
        if (h_ctl) cudaFreeHost(h_ctl);
        for (cudaStream_t s : aux_stream)
            if (s) cudaStreamDestroy(s);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

std::mutex g_mutex;
std::map<int, std::unique_ptr<Context>> g_ctx;
int g_next = 0;
std::string g_err;
bool g_configured[64] = {false};

Context* get_ctx(int h) {
    std::lock_guard<std::mutex> lk(g_mutex);
    auto it = g_ctx.find(h);
    return it == g_ctx.end() ? nullptr : it->second.get();
}

int fail(Context* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_err = msg;
    return code;
}

int cuda_fail(Context* c, cudaError_t e, const char* where) {
    return fail(c, GDFV_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Block, (i, j, k) and cell-centre position of the cell at global index g (the
// cell id of the reference's SFluidBlock is i + nic (j + njc k)).
bool locate_cell(const Context* c, long long g, int* blk, int* ijk, double* pos) {
    if (g < 0 || g >= c->total) return false;
    for (size_t b = 0; b < c->blocks.size(); ++b) {
        const HostBlock& hb = c->blocks[b];
        const long long n = (long long)hb.n[0] * hb.n[1] * hb.n[2];
        if (g < hb.offset || g >= hb.offset + n) continue;
        const long long id = g - hb.offset;
        const int ii[3] = {(int)(id % hb.n[0]), (int)((id / hb.n[0]) % hb.n[1]), (int)(id / ((long long)hb.n[0] * hb.n[1]))};
        if (blk) *blk = (int)b;
        for (int d = 0; d < 3; ++d) {
            if (ijk) ijk[d] = ii[d];
            if (pos) pos[d] = hb.origin[d] + ((double)ii[d] + 0.5) * hb.len[d];
        }
        if (pos && c->cfg.dims == 2) pos[2] = 0.0;
        return true;
    }
    return false;
}

// Records the failing cell of a failed step and describes it as the reference's
// decode failure and invalid-cell report do (e4/fvcell.d:610-640: block id, cell id,
// position; e4/fluidblock.d:607-675).
std::string bad_cell_text(Context* c, long long g) {
    int blk = 0, ijk[3] = {0, 0, 0};
    double pos[3] = {0.0, 0.0, 0.0};
    if (!locate_cell(c, g, &blk, ijk, pos)) { c->last_bad_cell = -1; return ""; }
    c->last_bad_cell = g;
    const HostBlock& hb = c->blocks[blk];
    const long long id = ijk[0] + (long long)hb.n[0] * (ijk[1] + (long long)hb.n[1] * ijk[2]);
    char buf[256];
    std::snprintf(buf, sizeof buf, " First bad cell: blk-id= %d cell-id= %lld (i,j,k)= (%d,%d,%d) x= %.17g y= %.17g z= %.17g",
                  blk, id, ijk[0], ijk[1], ijk[2], pos[0], pos[1], pos[2]);
    return buf;
}

#define CK(call)                                                      \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call);        \
    } while (0)

std::string norm(const char* s) {
    std::string r(s ? s : "");
    for (auto& ch : r) if (ch == '-') ch = '_';
    return r;
}

StageArgs stage_args(Context* c) {
    StageArgs A{};
    A.blocks = c->d_blocks;
    A.tiles = c->d_tiles;
    A.inflow = c->d_inflow;
    A.rot = c->d_rot;
    A.Ubuf[0] = c->U[0];
    A.Ubuf[1] = c->U[1];
    A.U_in = nullptr;
    A.dU0 = c->dU0;
    A.R_out = nullptr;
    A.ctl = c->d_ctl;
    A.max_signal = c->d_maxsig;
    A.last_signal = c->d_lastsig;
    A.total = c->total;
    A.P = c->P;
    A.n_tiles = c->n_tiles;
    A.n_tiles2 = c->n_tiles2;
    A.n_prim_wide = c->n_prim_wide;
    A.n_prim_narrow = c->n_prim_narrow;
    A.max_invalid_cells = c->cfg.max_invalid_cells;
    A.persistent = c->cfg.persistent;
    return A;
}

// Arguments of the context's own stepping (gdfv_run, the autotuner, gdfv_time_stages):
// with the float Euler path, the primitive buffers of the state buffers it steps
// (state_parity: which of U[0], U[1] the control record's step parity 0 names).
StageArgs stage_args_run(Context* c, int state_parity = 0) {
    StageArgs A = stage_args(c);
    if (c->prim[0]) {
        A.prim[0] = c->prim[state_parity];
        A.prim[1] = c->prim[state_parity ^ 1];
        A.prim1 = c->prim1;
    }
    return A;
}

int read_ctl(Context* c);

// Primitives of the current state for the kernels on decoded primitives, when the
// state was set from outside a stage since they were last made.
int ensure_prims(Context* c) {
    if (!c->prim[0] || c->prims_valid) return GDFV_OK;
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    const int parity = c->h_ctl->step & 1;
    prims_fp32(c->U[parity], c->total, c->P, c->prim[parity], c->stream);
    CK(cudaGetLastError());
    c->prims_valid = true;
    return GDFV_OK;
}

cudaError_t launch_stage(Context* c, int stage, const StageArgs& A) {
    if (c->cfg.precision == 0) return launch_stage_fp64(stage, c->cfg.flux, c->cfg.mhd, A, c->stream);
    return launch_stage_fp32(stage, c->cfg.flux, c->cfg.mhd, A, c->stream);
}

cudaError_t enqueue_step(Context* c) {
    StageArgs A = stage_args_run(c);
    step_begin_kernel<<<1, 1, 0, c->stream>>>(c->d_ctl, c->d_blocks, c->d_maxsig, c->d_lastsig, c->sp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = launch_stage(c, 1, A)) != cudaSuccess) return e;
    if ((e = launch_stage(c, 2, A)) != cudaSuccess) return e;
    step_end_kernel<<<1, 1, 0, c->stream>>>(c->d_ctl, c->sp);
    return cudaGetLastError();
}

// Scratch of the fixed-dt steps and the autotuner's trial steps (control record,
// signal maxima), and of the MHD step adjoint's signal scans; allocated on first use.
int step_scratch(Context* c) {
    if (c->step_ctl) return 0;
    const size_t nb = c->blocks.size();
    if (cudaMalloc(&c->step_ctl, sizeof(Control)) != cudaSuccess ||
        cudaMalloc(&c->step_maxsig, sizeof(unsigned long long) * nb) != cudaSuccess ||
        cudaMalloc(&c->step_lastsig, sizeof(double) * nb) != cudaSuccess ||
        cudaMalloc(&c->ch_maxsig, sizeof(unsigned long long) * nb) != cudaSuccess ||
        cudaMalloc(&c->ch_lastsig, sizeof(double) * nb) != cudaSuccess ||
        cudaMalloc(&c->ch_bad, sizeof(int)) != cudaSuccess) {
        fail(c, GDFV_ERR_CUDA, "cudaMalloc of the step scratch failed");
        return 1;
    }
    return 0;
}

// Per-block signal maxima of the current state (needed by the first dt check).
int scan_signal(Context* c) {
    CK(cudaMemsetAsync(c->d_maxsig, 0, sizeof(unsigned long long) * c->blocks.size(), c->stream));
    CK(cudaMemsetAsync(c->d_bad, 0, sizeof(int), c->stream));
    CK(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const double* Ucur = c->U[c->h_ctl->step & 1];
    for (size_t b = 0; b < c->blocks.size(); ++b) {
        long long n = (long long)c->blocks[b].n[0] * c->blocks[b].n[1] * c->blocks[b].n[2];
        int nb = (int)((n + 255) / 256);
        signal_scan_kernel<<<nb, 256, 0, c->stream>>>(Ucur, c->total, c->d_blocks, (int)b, c->P, c->d_maxsig,
                                                       c->d_lastsig, c->d_bad);
        CK(cudaGetLastError());
    }
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, c->d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (bad) return fail(c, GDFV_ERR_ARG, "state contains cells that do not decode");
    c->signal_valid = true;
    return GDFV_OK;
}

// Per-block signal maxima of the state U into maxsig, enqueued on s (no host
// synchronisation; cells that do not decode are counted in *bad and left out).
cudaError_t enqueue_signal_scan(Context* c, cudaStream_t s, const double* U, unsigned long long* maxsig,
                                double* lastsig, int* bad) {
    cudaError_t e = cudaMemsetAsync(maxsig, 0, sizeof(unsigned long long) * c->blocks.size(), s);
    for (size_t b = 0; b < c->blocks.size() && e == cudaSuccess; ++b) {
        const long long n = (long long)c->blocks[b].n[0] * c->blocks[b].n[1] * c->blocks[b].n[2];
        signal_scan_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(U, c->total, c->d_blocks, (int)b, c->P, maxsig,
                                                                        lastsig, bad);
        e = cudaGetLastError();
    }
    return e;
}

void fill_weights(double len, double* w) {
    // e4/onedinterp.d:338-355 l2r2_prepare with all four lengths equal
    const double lenL1 = len, lenL0 = len, lenR0 = len, lenR1 = len;
    w[W_LENL0] = lenL0;
    w[W_LENR0] = lenR0;
    w[W_AL0] = 0.5 * lenL0 / (lenL1 + 2.0 * lenL0 + lenR0);
    w[W_AR0] = 0.5 * lenR0 / (lenL0 + 2.0 * lenR0 + lenR1);
    w[W_TOL] = 2.0 / (lenL0 + lenL1);
    w[W_TOC] = 2.0 / (lenR0 + lenL0);
    w[W_TOR] = 2.0 / (lenR1 + lenR0);
    w[W_TWOL] = (2.0 * lenL0 + lenL1);
    w[W_TWOR] = (2.0 * lenR0 + lenR1);
}

// Tile table over all blocks: 32 x TJ columns and kchunk planes per tile (0: the
// block's nkc up to 32).  Ordered by decreasing work (cells), so that a grid
// taking tiles in order -- the hardware's CTA order, or the persistent stride --
// starts the long tiles of uneven blocks first.
// Tiles of TI x TJ cells (k chunks of kchunk planes) over the i strips (i0 a multiple of
// TI) that pick(block, i0) selects, sorted by decreasing work.
template <class Pick>
void build_tiles_strips(Context* c, int kchunk, int TI, int TJ, Pick pick, std::vector<TileDesc>& tiles) {
    tiles.clear();
    for (size_t b = 0; b < c->blocks.size(); ++b) {
        const HostBlock& hb = c->blocks[b];
        int kc = kchunk > 0 ? kchunk : std::min(hb.n[2], 32);
        if (c->cfg.dims == 2) kc = 1;
        for (int k0 = 0; k0 < hb.n[2]; k0 += kc)
            for (int j0 = 0; j0 < hb.n[1]; j0 += TJ)
                for (int i0 = 0; i0 < hb.n[0]; i0 += TI) {
                    if (!pick(hb, i0)) continue;
                    TileDesc t{};
                    t.block = (int)b; t.i0 = i0; t.j0 = j0; t.k0 = k0; t.k1 = std::min(k0 + kc, hb.n[2]);
                    tiles.push_back(t);
                }
    }
    auto work = [&](const TileDesc& t) {
        const HostBlock& hb = c->blocks[t.block];
        return (long long)std::min(TI, hb.n[0] - t.i0) * std::min(TJ, hb.n[1] - t.j0) * (t.k1 - t.k0);
    };
    std::stable_sort(tiles.begin(), tiles.end(), [&](const TileDesc& a, const TileDesc& b) { return work(a) > work(b); });
}

void build_tiles_rows(Context* c, int kchunk, int TJ, std::vector<TileDesc>& tiles) {
    build_tiles_strips(c, kchunk, 32, TJ, [](const HostBlock&, int) { return true; }, tiles);
}

// Fraction of the tile rows of all blocks that hold cells, weighted by cells per row.
double row_use(const Context* c, int TJ) {
    double used = 0.0, slots = 0.0;
    for (const HostBlock& hb : c->blocks) {
        const double w = (double)hb.n[0] * hb.n[2];
        used += w * hb.n[1];
        slots += w * (double)((hb.n[1] + TJ - 1) / TJ) * TJ;
    }
    return slots > 0.0 ? used / slots : 1.0;
}

// The tile table of a run: stages 0 and 1, then -- when the corrector has other rows
// and they pay off -- the corrector's own table.  n1 and n2 receive their lengths
// (n2 = 0: the corrector runs over the first table).  The float Euler corrector runs
// about 6% faster per tile slot with its 7 rows (more registers per thread at the same
// CTAs per SM) than with 8 on a 256^3 block, but not on small blocks, where the
// four-plane prologue of each tile weighs more: a 64-block lattice of 32-128 rows with
// 96% row use ran 2.5% slower.  So the corrector gets its own table only when its rows
// leave at most about 3% more empty row slots than the shared ones.
//
// The kernel on decoded primitives (float Euler defaults) takes tiles 32 or 16 cells wide
// (GeoF; 16 wide: two rows per warp, twice the rows), by cfg.tile_width.  With 16 its
// table follows the others: n3 = 0 tiles 32 wide, n4 tiles 16 wide.  n3 = n4 = 0: it runs
// over the first table.  The other kernels (and the no-alloc step, which runs them) keep
// the first tables.  (Both widths in one stage, 16-wide tiles only for the strip left at
// a block's i end, ran slower: the second, small launch waits for the first to drain.)
void build_tiles(Context* c, int kchunk, std::vector<TileDesc>& tiles, int& n1, int& n2, int& n3, int& n4) {
    const int TJ = tile_rows(c->cfg.precision, c->cfg.mhd);
    build_tiles_rows(c, kchunk, TJ, tiles);
    n1 = (int)tiles.size();
    n2 = n3 = n4 = 0;
    const int TJ2 = tile_rows_corrector(c->cfg.precision, c->cfg.mhd);
    if (TJ2 != TJ && row_use(c, TJ2) * 1.03 > row_use(c, TJ)) {
        std::vector<TileDesc> t2;
        build_tiles_rows(c, kchunk, TJ2, t2);
        n2 = (int)t2.size();
        tiles.insert(tiles.end(), t2.begin(), t2.end());
    }
    if (!(c->cfg.precision == 1 && prim_path(c->P)) || c->cfg.tile_width != 16) return;
    std::vector<TileDesc> t4;
    build_tiles_strips(c, kchunk, 16, 2 * TJ, [](const HostBlock&, int) { return true; }, t4);
    n4 = (int)t4.size();
    tiles.insert(tiles.end(), t4.begin(), t4.end());
}

// The cell that feeds each ghost of an ExchangeBC_FullFace, as a map word: for the
// partner's index along axis d, bits 3d..3d+1 select this block's i, j, k or the ghost's
// depth (0..3), and bit 3d+2 counts it from the partner's far end.
// GhostCellFullFaceCopy.set_up_cell_mapping_phase0 (e4/bc/ghost_cell_effect/
// full_face_copy.d:680-1409) spells it out for 6 x 6 face pairs and 4 orientations;
// every case there follows one rule, restated here.  Each face has
// a tangential frame of two axes with signs, right-handed about its outward normal:
// west (-j, k), east (j, k), south (i, k), north (-i, k), bottom (-i, j), top (i, j).
// Seen from the partner the ghost's frame is mirrored (first axis reversed), then turned
// by `orientation` quarter turns ((a, b) -> (-b, a) each); its coordinates are then the
// source's coordinates in the partner face's frame.  Along the partner's normal the
// source lies `depth` cells inside the face.  2D blocks take orientation 0, as there.
const int kFaceAxis[6][2] = {{1, 2}, {1, 2}, {0, 2}, {0, 2}, {0, 1}, {0, 1}};
const int kFaceSign[6][2] = {{-1, 1}, {1, 1}, {1, 1}, {-1, 1}, {-1, 1}, {1, 1}};

int exchange_map(int dims, int face, int other_face, int orientation) {
    int ax[2] = {kFaceAxis[face][0], kFaceAxis[face][1]};
    int sg[2] = {-kFaceSign[face][0], kFaceSign[face][1]};
    const int turns = dims == 2 ? 0 : orientation;
    for (int t = 0; t < turns; ++t) {
        const int a0 = ax[0], s0 = sg[0];
        ax[0] = ax[1]; sg[0] = -sg[1];
        ax[1] = a0; sg[1] = s0;
    }
    int sel[3], flip[3];
    sel[other_face / 2] = 3;
    flip[other_face / 2] = other_face & 1;
    for (int r = 0; r < 2; ++r) {
        const int d = kFaceAxis[other_face][r];
        sel[d] = ax[r];
        flip[d] = kFaceSign[other_face][r] * sg[r] < 0;
    }
    int xm = 0;
    for (int d = 0; d < 3; ++d) xm |= (sel[d] | (flip[d] << 2)) << (3 * d);
    return xm;
}

// The map as the kernels evaluate it: partner cell = x[0] + x[1] i + x[2] j + x[3] k for
// the ghost (i, j, k) beyond face `face` (depth = -1 - index on a minus face, index - n
// on a plus face).  Block cell counts are below 2^31, so the coefficients fit an int.
void exchange_linear(int xm, int face, const int* n, const int* on, int* x) {
    const int ax = face / 2, plus = face & 1;
    const long long stride[3] = {1, (long long)on[0], (long long)on[0] * on[1]};
    long long c[4] = {0, 0, 0, 0};
    for (int d = 0; d < 3; ++d) {
        const int sel = (xm >> (3 * d)) & 3, flip = (xm >> (3 * d + 2)) & 1;
        // v = a + b * (this block's index along axis `src`)
        const int src = sel == 3 ? ax : sel;
        long long a = 0, b = 1;
        if (sel == 3) { a = plus ? -(long long)n[ax] : -1; b = plus ? 1 : -1; }
        // p = flip ? on[d] - 1 - v : v
        long long pa = flip ? on[d] - 1 - a : a, pb = flip ? -b : b;
        c[0] += stride[d] * pa;
        c[1 + src] += stride[d] * pb;
    }
    // kept modulo 2^32: the kernels evaluate the sum in 32-bit wrap-around arithmetic
    for (int m = 0; m < 4; ++m) x[m] = (int)(unsigned)(unsigned long long)c[m];
}

int do_prepare(Context* c) {
    Config& g = c->cfg;
    if (c->blocks.empty()) return fail(c, GDFV_ERR_STATE, "no blocks");
    if (g.flux == FLUX_HLLE && !g.mhd) return fail(c, GDFV_ERR_ARG, "hlle is the MHD flux: set MHD=1");
    if (g.mhd && g.flux != FLUX_HLLE) return fail(c, GDFV_ERR_ARG, "MHD runs use flux_calculator=hlle");
    if (g.dims != 2 && g.dims != 3) return fail(c, GDFV_ERR_ARG, "dimensions must be 2 or 3");
    c->nq = g.mhd ? 10 : 5;
    const int nfaces = g.dims == 3 ? 6 : 4;
    long long off = 0;
    std::vector<InflowState> inflows;
    struct FixedState { int block, face; InflowState state; };
    std::vector<FixedState> fixed;
    std::vector<double> rots;   // Rmatrix of each rotating exchange face
    int outflow_bcs = 0;
    c->h_blocks.clear();
    c->h_inflow.clear();
    std::vector<TileDesc> tiles;
    const double Cv = g.R / (g.gamma - 1.0);
    for (size_t b = 0; b < c->blocks.size(); ++b) {
        HostBlock& hb = c->blocks[b];
        if (g.dims == 2 && hb.n[2] != 1) return fail(c, GDFV_ERR_ARG, "2D blocks have nkc = 1");
        for (int d = 0; d < (g.dims == 3 ? 3 : 2); ++d)
            if (hb.n[d] < 2) return fail(c, GDFV_ERR_ARG, "blocks need at least 2 cells per active direction");
        // the kernels index cells (and the adjoint faces of one direction) within a
        // block in 32-bit arithmetic
        if ((long long)(hb.n[0] + 1) * (hb.n[1] + 1) * (hb.n[2] + 1) > 2147483647LL)
            return fail(c, GDFV_ERR_ARG, "a block has more than 2^31 - 1 cells or faces (split it into several blocks)");
        hb.offset = off;
        BlockDesc B{};
        for (int d = 0; d < 3; ++d) { B.n[d] = hb.n[d]; B.len[d] = hb.len[d]; fill_weights(hb.len[d], B.w[d]); }
        B.offset = off;
        if (g.dims == 2) {
            B.area[0] = hb.len[1]; B.area[1] = hb.len[0]; B.area[2] = 0.0;
            B.vol_inv = 1.0 / (hb.len[0] * hb.len[1]);
            B.L_min = std::min(hb.len[0], hb.len[1]);
        } else {
            B.area[0] = hb.len[1] * hb.len[2];
            B.area[1] = hb.len[2] * hb.len[0];
            B.area[2] = hb.len[0] * hb.len[1];
            B.vol_inv = 1.0 / (hb.len[0] * hb.len[1] * hb.len[2]);
            B.L_min = std::min(std::min(hb.len[0], hb.len[1]), hb.len[2]);
        }
        B.x0 = hb.origin[0]; B.y0 = hb.origin[1]; B.z0 = hb.origin[2];
        for (int f = 0; f < 6; ++f) {
            const HostBC& bc = hb.bc[f];
            B.bc_type[f] = bc.type;
            B.bc_xorder[f] = bc.x_order;
            B.bc_other[f] = bc.other;
            B.bc_other_face[f] = bc.other_face;
            B.bc_inflow[f] = -1;
            if (f >= nfaces) continue;
            for (int m = 0; m < 4; ++m) B.bc_xlin[f][m] = 0;
            B.bc_xrot[f] = 0;
            if (bc.type == BC_EXCHANGE) {
                if (bc.other < 0 || bc.other >= (int)c->blocks.size())
                    return fail(c, GDFV_ERR_ARG, "exchange partner block does not exist");
                if (bc.other_face < 0 || bc.other_face >= nfaces)
                    return fail(c, GDFV_ERR_ARG, "exchange partner face does not exist");
                if (bc.orientation < 0 || bc.orientation > 3)
                    return fail(c, GDFV_ERR_ARG, "exchange orientation must be 0..3");
                const HostBlock& ob = c->blocks[bc.other];
                const int xm = exchange_map(g.dims, f, bc.other_face, bc.orientation);
                for (int d = 0; d < 3; ++d) {
                    const int sel = (xm >> (3 * d)) & 3;
                    if (sel < 3 && ob.n[d] != hb.n[sel])
                        return fail(c, GDFV_ERR_ARG, "exchange faces differ in size (block " + std::to_string(b) +
                                                         " face " + std::to_string(f) + ")");
                }
                if (ob.n[bc.other_face / 2] < 2) return fail(c, GDFV_ERR_ARG, "exchange partner is too thin");
                exchange_linear(xm, f, hb.n, ob.n, B.bc_xlin[f]);
                if (bc.rotate) {
                    B.bc_xrot[f] = (int)(1 + rots.size() / 9);
                    rots.insert(rots.end(), bc.rot, bc.rot + 9);
                }
            }
            if (bc.type == BC_EXTRAPOLATE && (bc.x_order < 0 || bc.x_order > 1))
                return fail(c, GDFV_ERR_ARG, "x_order must be 0 or 1");
            if (bc.type == BC_SIMPLE_FLUX && g.mhd)
                return fail(c, GDFV_ERR_ARG, "outflow_simple_flux is not defined for MHD (boundary_flux_effect.d:519)");
            if (bc.type == BC_FIXED_P || bc.type == BC_FIXED_PT || bc.type == BC_SIMPLE_FLUX) outflow_bcs = 1;
            if (bc.type == BC_FIXED_P || bc.type == BC_FIXED_PT) {
                // the outside state of fixed_p.d / fixed_pt.d: p (and rho = p/(T R), u = Cv T)
                InflowState s{};
                s.p = bc.inflow[0];
                if (bc.type == BC_FIXED_PT) {
                    s.rho = bc.inflow[0] / (bc.inflow[1] * g.R);
                    s.u = Cv * bc.inflow[1];
                }
                fixed.push_back({(int)b, f, s});
            }
            if (bc.type == BC_INFLOW) {
                // FlowState:new{p=, T=, ...}: update_thermo_from_pT + update_sound_speed
                InflowState s{};
                double p = bc.inflow[0], T = bc.inflow[1];
                if (!(p > 0.0) || !(T > 0.0)) return fail(c, GDFV_ERR_ARG, "inflow needs p > 0 and T > 0");
                s.p = p;
                s.rho = p / (T * g.R);
                s.u = Cv * T;
                s.a = std::sqrt(g.gamma * g.R * T);
                for (int d = 0; d < 3; ++d) { s.vel[d] = bc.inflow[2 + d]; s.B[d] = bc.inflow[5 + d]; }
                s.psi = bc.inflow[8];
                B.bc_inflow[f] = (int)inflows.size();
                inflows.push_back(s);
                c->h_inflow.insert(c->h_inflow.end(), bc.inflow, bc.inflow + 9);
            }
        }
        c->h_blocks.push_back(B);
        off += (long long)hb.n[0] * hb.n[1] * hb.n[2];
    }
    // outside states of the fixed-p boundaries after the supersonic-inflow states
    c->n_inflow = (int)inflows.size();
    for (const FixedState& fx : fixed) {
        c->h_blocks[fx.block].bc_inflow[fx.face] = (int)inflows.size();
        inflows.push_back(fx.state);
    }
    c->total = off;
    // graded blocks: cell lengths of cells -2 .. n+1 per direction (ghosts: the partner's
    // cells across an exchange face, else the block's own interior cell n, as SFluidBlock
    // gives them, e4/sfluidblock.d:884-1090, simcore_exchange.d:44-70) and the l2r2 weights
    // of cells -1 .. n; one device buffer for all of them
    std::vector<double> geom;
    std::vector<std::array<long long, 6>> geom_at(c->blocks.size());
    int any_graded = 0;
    for (size_t b = 0; b < c->blocks.size(); ++b) {
        const HostBlock& hb = c->blocks[b];
        if (!hb.graded()) continue;
        any_graded = 1;
        if (g.mhd) return fail(c, GDFV_ERR_ARG, "graded blocks are not offered with MHD");
        if (g.lmr_epsilon) return fail(c, GDFV_ERR_ARG, "graded blocks are not offered with van_albada_variant lmr");
        double lmin[3];
        for (int d = 0; d < 3; ++d) {
            const int n = hb.n[d];
            std::vector<double> L((size_t)n + 4);
            for (int cc = 0; cc < n; ++cc) L[(size_t)cc + 2] = hb.cell_len(d, cc);
            lmin[d] = *std::min_element(L.begin() + 2, L.begin() + 2 + n);
            for (int side = 0; side < 2; ++side) {
                const HostBC& bc = hb.bc[2 * d + side];
                for (int m = 0; m < 2; ++m) {
                    double v;
                    if (bc.type == BC_EXCHANGE && 2 * d + side < nfaces) {
                        // the partner's cell m layers inside its face, along its normal
                        const HostBlock& ob = c->blocks[bc.other];
                        const int od = bc.other_face / 2;
                        v = ob.cell_len(od, (bc.other_face & 1) ? ob.n[od] - 1 - m : m);
                    } else {
                        v = hb.cell_len(d, side ? n - 1 - m : m);
                    }
                    L[(size_t)(side ? n + m : -1 - m) + 2] = v;
                }
            }
            geom_at[b][d] = (long long)geom.size();
            geom.insert(geom.end(), L.begin(), L.end());
            geom_at[b][3 + d] = (long long)geom.size();
            for (int cc = -1; cc <= n; ++cc) {
                const double lm = L[(size_t)cc + 1], l0 = L[(size_t)cc + 2], lp = L[(size_t)cc + 3];
                // l2r2_prepare (e4/onedinterp.d:338-355) of faces c+1/2 and c-1/2
                const double wv[GW_N] = {2.0 / (l0 + lm), 2.0 / (lp + l0), 0.5 * l0 / (lm + 2.0 * l0 + lp),
                                         2.0 * l0 + lm, lp, lm, 2.0 * l0 + lp};
                geom.insert(geom.end(), wv, wv + GW_N);
            }
        }
        BlockDesc& B = c->h_blocks[b];
        B.graded = 1;
        B.x0 = hb.vert[0][0]; B.y0 = hb.vert[1][0]; B.z0 = hb.vert[2][0];
        B.L_min = g.dims == 3 ? std::min(std::min(lmin[0], lmin[1]), lmin[2]) : std::min(lmin[0], lmin[1]);
    }
    NumParams& P = c->P;
    P.gas.R = g.R; P.gas.gamma = g.gamma; P.gas.Cv = Cv; P.gas.Cvinv = 1.0 / Cv;
    P.eps_van_albada = g.eps_van_albada;
    P.divB_damping_length = g.divB_damping_length;
    P.max_velocity = g.max_velocity; P.max_temp = g.max_temp; P.min_temp = g.min_temp;
    P.apply_limiter = g.apply_limiter; P.extrema_clipping = g.extrema_clipping;
    P.apply_entropy_fix = g.apply_entropy_fix; P.glm_reference_indexing = g.glm_reference_indexing;
    P.mhd = g.mhd; P.divergence_cleaning = g.divergence_cleaning; P.dims = g.dims;
    P.stringent_cfl = g.stringent_cfl; P.nq = c->nq; P.lmr_epsilon = g.lmr_epsilon;
    P.outflow_bcs = outflow_bcs;
    P.graded = any_graded;
    P.rotating = !rots.empty();
    StepParams& sp = c->sp;
    sp.cfl_count = g.cfl_count; sp.n_stages = 2; sp.fixed_time_step = g.fixed_time_step;
    sp.mhd_cleaning = g.mhd && g.divergence_cleaning;
    sp.max_attempts = g.max_attempts; sp.max_invalid_cells = g.max_invalid_cells;
    sp.nblocks = (int)c->blocks.size();
    sp.cfl_value = g.cfl_value; sp.dt_init = g.dt_init; sp.dt_max = g.dt_max;
    // (after the options: the tables depend on which kernels run)
    build_tiles(c, g.tile_kchunk, tiles, c->n_tiles, c->n_tiles2, c->n_prim_wide, c->n_prim_narrow);

    CK(cudaGetDevice(&c->device));
    if (c->device < 64 && !g_configured[c->device]) {
        CK(configure_stage_fp64());
        CK(configure_stage_fp32());
        g_configured[c->device] = true;
    }
    if (!c->stream) {
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    const size_t bytes = sizeof(double) * (size_t)c->nq * (size_t)c->total;
    CK(cudaMalloc(&c->U[0], bytes));
    CK(cudaMalloc(&c->U[1], bytes));
    CK(cudaMalloc(&c->dU0, bytes));
    CK(cudaMemset(c->U[0], 0, bytes));
    CK(cudaMemset(c->U[1], 0, bytes));
    CK(cudaMemset(c->dU0, 0, bytes));
    // the float form runs the kernel on decoded primitives; the FP64 form ran it bit for bit
    // but slower than stage_kernel (2,071 against 2,164 Mcell-updates/s at 256^3)
    if (g.precision == 1 && prim_path(c->P)) {
        const size_t pbytes = sizeof(float) * 6 * (size_t)c->total;
        CK(cudaMalloc(&c->prim[0], pbytes));
        CK(cudaMalloc(&c->prim[1], pbytes));
        CK(cudaMalloc(&c->prim1, pbytes));
    }
    c->prims_valid = false;
    if (!geom.empty()) {
        CK(cudaMalloc(&c->d_geom, sizeof(double) * geom.size()));
        CK(cudaMemcpy(c->d_geom, geom.data(), sizeof(double) * geom.size(), cudaMemcpyHostToDevice));
        for (size_t b = 0; b < c->h_blocks.size(); ++b) {
            if (!c->h_blocks[b].graded) continue;
            for (int d = 0; d < 3; ++d) {
                c->h_blocks[b].glen[d] = c->d_geom + geom_at[b][d];
                c->h_blocks[b].gw[d] = c->d_geom + geom_at[b][3 + d];
            }
        }
    }
    if (!rots.empty()) {
        CK(cudaMalloc(&c->d_rot, sizeof(double) * rots.size()));
        CK(cudaMemcpy(c->d_rot, rots.data(), sizeof(double) * rots.size(), cudaMemcpyHostToDevice));
    }
    CK(cudaMalloc(&c->d_blocks, sizeof(BlockDesc) * c->h_blocks.size()));
    CK(cudaMemcpy(c->d_blocks, c->h_blocks.data(), sizeof(BlockDesc) * c->h_blocks.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_tiles, sizeof(TileDesc) * tiles.size()));
    c->tiles_cap = tiles.size();
    CK(cudaMemcpy(c->d_tiles, tiles.data(), sizeof(TileDesc) * tiles.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_inflow, sizeof(InflowState) * std::max<size_t>(1, inflows.size())));
    if (!inflows.empty())
        CK(cudaMemcpy(c->d_inflow, inflows.data(), sizeof(InflowState) * inflows.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_ctl, sizeof(Control)));
    CK(cudaMallocHost(&c->h_ctl, sizeof(Control)));
    std::memset(c->h_ctl, 0, sizeof(Control));
    c->h_ctl->dt_global = g.dt_init;  // e4/simcore.d:761
    c->h_ctl->first_bad_cell = LLONG_MAX;
    CK(cudaMemcpy(c->d_ctl, c->h_ctl, sizeof(Control), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_maxsig, sizeof(unsigned long long) * c->blocks.size()));
    CK(cudaMalloc(&c->d_lastsig, sizeof(double) * c->blocks.size()));
    CK(cudaMalloc(&c->d_bad, sizeof(int)));
    CK(cudaMemset(c->d_maxsig, 0, sizeof(unsigned long long) * c->blocks.size()));
    CK(cudaMemset(c->d_lastsig, 0, sizeof(double) * c->blocks.size()));
    c->prepared = true;
    return GDFV_OK;
}

int read_ctl(Context* c) {
    CK(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GDFV_OK;
}

int write_ctl(Context* c) {
    CK(cudaMemcpyAsync(c->d_ctl, c->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GDFV_OK;
}

constexpr int kGraphSteps = 8;

void drop_graphs(Context* c) {
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    if (c->graph1) { cudaGraphExecDestroy(c->graph1); c->graph1 = nullptr; }
}

// The step slots of a run, captured once: kGraphSteps of them, and one alone for the
// tail of a run (a slot past the halt is a no-op, but still launches its kernels).
int build_graph(Context* c) {
    drop_graphs(c);
    for (int n : {kGraphSteps, 1}) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int s = 0; s < n && e == cudaSuccess; ++s) e = enqueue_step(c);
        cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
        if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(c, e, "capture step"); }
        if (e2 != cudaSuccess) return cuda_fail(c, e2, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(n == 1 ? &c->graph1 : &c->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
    }
    c->graph_steps = kGraphSteps;
    return GDFV_OK;
}

// Read-only view of a context for gdfv_step_noalloc (gdfv_noalloc.cu).

bool noalloc_view(int ctx, NoallocView* v) {
    Context* c = get_ctx(ctx);
    if (!c || !v) return false;
    v->prepared = c->prepared;
    v->precision = c->cfg.precision;
    v->flux = c->cfg.flux;
    v->mhd = c->cfg.mhd;
    v->nblocks = (int)c->blocks.size();
    v->max_invalid_cells = c->cfg.max_invalid_cells;
    v->total = c->total;
    v->nq = c->nq;
    v->n_tiles = c->n_tiles;
    v->n_tiles2 = c->n_tiles2;
    v->d_blocks = c->d_blocks;
    v->d_tiles = c->d_tiles;
    v->d_inflow = c->d_inflow;
    v->d_rot = c->d_rot;
    v->P = c->P;
    v->c_h = c->h_ctl ? c->h_ctl->c_h : 0.0;
    v->stream = c->stream;
    v->persistent = c->cfg.persistent;
    v->max_block_cells = 0;
    for (const HostBlock& hb : c->blocks)
        v->max_block_cells = std::max(v->max_block_cells, (long long)hb.n[0] * hb.n[1] * hb.n[2]);
    return true;
}

void noalloc_set_error(int ctx, const std::string& msg) {
    Context* c = get_ctx(ctx);
    if (c) c->err = msg;
    else g_err = msg;
}

std::string noalloc_bad_cell_text(int ctx, long long g) {
    Context* c = get_ctx(ctx);
    return c ? bad_cell_text(c, g) : std::string();
}

bool adjoint_view(int ctx, AdjView* v) {
    Context* c = get_ctx(ctx);
    if (!c || !v) return false;
    v->prepared = c->prepared;
    v->flux = c->cfg.flux;
    v->mhd = c->cfg.mhd;
    v->precision = c->cfg.precision;
    v->nblocks = (int)c->blocks.size();
    v->ninflow = c->n_inflow;
    v->dims = c->cfg.dims;
    v->total = c->total;
    v->d_blocks = c->d_blocks;
    v->d_inflow = c->d_inflow;
    v->d_rot = c->d_rot;
    v->P = c->P;
    v->c_h = c->h_ctl ? c->h_ctl->c_h : 0.0;
    v->stream = c->stream;
    v->h_blocks = c->h_blocks;
    v->scratch = &c->adj_scratch;
    v->scratch_n = &c->adj_scratch_n;
    v->scratch_ready = &c->adj_ready;
    return true;
}

void adjoint_set_error(int ctx, const std::string& msg) {
    Context* c = get_ctx(ctx);
    if (c) c->err = msg;
    else g_err = msg;
}

// U1 = U0 + dt*dU0 with the predictor's rounding (no contraction), MHD psi not damped:
// used only for the Euler adjoint.
__global__ void predictor_state_kernel(const double* U0, const double* dU0, double dt, long long n, double* U1) {
    long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < n) U1[x] = __dadd_rn(U0[x], __dmul_rn(dt, dU0[x]));
}

// Record of the step that just completed (gdfv_run_record): the state after it (the
// buffer the step counter's parity names), its predictor state U0 + dt dU0 (U0 in the
// other buffer, the step's input, in the predictor's operation order) and its dt.  A step
// counter other than `expect` means the step did not complete in its slot (a retry, or a
// failure): *flag is set and nothing is written.
__global__ void record_step_kernel(const Control* ctl, const double* U0buf, const double* U1buf, const double* dU0,
                                   long long n, int expect, double* state_out, double* pred_out, double* dt_out,
                                   int* flag) {
    if (ctl->step != expect || ctl->status != ST_OK) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *flag = 1;
        return;
    }
    const double* cur = (ctl->step & 1) ? U1buf : U0buf;
    const double* prev = (ctl->step & 1) ? U0buf : U1buf;
    const double dt = ctl->dt_global;
    if (blockIdx.x == 0 && threadIdx.x == 0) *dt_out = dt;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x) {
        if (state_out) state_out[x] = cur[x];
        if (pred_out) pred_out[x] = __dadd_rn(prev[x], __dmul_rn(dt, dU0[x]));
    }
}

// Residual norms of dU/dt (e4/fluidblock.d:861-909): per CTA, the maximum of |dU/dt[q]|
// for every q and the sum of squares of the quantities compute_L2_residual takes
// (mass, x and y momentum, z momentum in 3D, total energy, with MHD xB and yB).
// Grid-stride over cells, two cells per step (2 NQ loads in flight), warp shuffles,
// then the warps in order: partial[cta][NQ + 1].
constexpr int kNormThreads = 256;
template <int NQ>
__global__ void __launch_bounds__(kNormThreads) residual_norms_kernel(const double* __restrict__ dU, long long total,
                                                                       int threeD, double* partial) {
    double mx[NQ], l2 = 0.0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) mx[q] = 0.0;
    auto in_l2 = [&](int q) {
        return q == MASS || q == XMOM || q == YMOM || (q == ZMOM && threeD) || q == TOTENERGY || q == XB || q == YB;
    };
    const long long stride = (long long)gridDim.x * blockDim.x;
    long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (; x + stride < total; x += 2 * stride) {
        double a[NQ], b[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            a[q] = __ldg(dU + (long long)q * total + x);
            b[q] = __ldg(dU + (long long)q * total + x + stride);
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            mx[q] = fmax(mx[q], fmax(fabs(a[q]), fabs(b[q])));
            if (in_l2(q)) l2 += a[q] * a[q] + b[q] * b[q];
        }
    }
    if (x < total) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const double v = __ldg(dU + (long long)q * total + x);
            mx[q] = fmax(mx[q], fabs(v));
            if (in_l2(q)) l2 += v * v;
        }
    }
    __shared__ double s_part[kNormThreads / 32][NQ + 1];
    for (int o = 16; o > 0; o >>= 1) {
        l2 += __shfl_xor_sync(0xffffffffu, l2, o);
#pragma unroll
        for (int q = 0; q < NQ; ++q) mx[q] = fmax(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], o));
    }
    const int wv = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) s_part[wv][q] = mx[q];
        s_part[wv][NQ] = l2;
    }
    __syncthreads();
    if (threadIdx.x <= NQ) {
        const int q = threadIdx.x;
        double r = s_part[0][q];
        for (int w = 1; w < kNormThreads / 32; ++w) r = q == NQ ? r + s_part[w][q] : fmax(r, s_part[w][q]);
        partial[(long long)blockIdx.x * (NQ + 1) + q] = r;
    }
}

// The CTAs' partials, one warp per quantity in a fixed order: out[q] = max for q < nq,
// out[nq] = sqrt(sum) (e4/simcore.d:1212).  Launched with 32 (nq + 1) threads.
__global__ void residual_norms_final_kernel(const double* partial, int ncta, int nq, double* out) {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q > nq) return;
    const bool sum = q == nq;
    double r = 0.0;   // maxima of magnitudes start at 0
    for (int b = lane; b < ncta; b += 32) {
        const double v = partial[(long long)b * (nq + 1) + q];
        r = sum ? r + v : fmax(r, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double t = __shfl_xor_sync(0xffffffffu, r, o);
        r = sum ? r + t : fmax(r, t);
    }
    if (lane == 0) out[q] = sum ? sqrt(r) : r;
}

// Resets the control record of a single fixed-dt step.
__global__ void step_dt_begin_kernel(Control* c, unsigned long long* maxsig, int nblocks, double dt, double c_h) {
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

// Frechet JVP helpers (e4/steadystate_core.d:1878-1970, :3040-3078).
constexpr int kJvpSumBlocks = 592;   // 4 x 148 SMs
// Per-CTA partial sums of eps*|U| + eps and v*v (added on the host in CTA order).
__global__ void jvp_sums_kernel(const double* U, const double* v, long long n, double eps, double* partial) {
    __shared__ double s1[256], s2[256];
    double a = 0.0, b = 0.0;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x) {
        a += eps * fabs(U[x]) + eps;
        b += v[x] * v[x];
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) { s1[threadIdx.x] += s1[threadIdx.x + o]; s2[threadIdx.x] += s2[threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s1[0]; partial[2 * blockIdx.x + 1] = s2[0]; }
}

__global__ void jvp_axpy_kernel(const double* U, const double* v, double sigma, long long n, double* Up) {
    long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < n) Up[x] = U[x] + sigma * v[x];
}

__global__ void jvp_diff_kernel(const double* R1, const double* R0, double sigma, long long n, double* Jv) {
    long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (x < n) Jv[x] = (R1[x] - R0[x]) / sigma;
}

// Sets the dt of the next step of a gdfv_steps_dt chain; failure counts carry over.
__global__ void step_dt_next_kernel(Control* c, double dt) {
    c->dt_global = dt;
    c->step = 0;
}

// c_h of a step of dt from the per-block signal maxima of its start state, with the
// operations of step_begin_kernel (e4/simcore.d:1625-1648, e4/fluidblock.d:975-995);
// the maxima are cleared for the next reduction.
__device__ double ch_from_maxsig(const BlockDesc* blocks, unsigned long long* maxsig, int nblocks, double dt) {
    double c_h = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        const double smax = __longlong_as_double((long long)maxsig[b]);
        const double cfl_max = smax * dt;
        const double ch = cfl_max * blocks[b].L_min / dt;
        c_h = b == 0 ? ch : fmin(ch, c_h);
        maxsig[b] = 0ull;
    }
    return c_h;
}

// The next fixed-dt step of an MHD chain with divergence cleaning: dt and its c_h.
__global__ void step_dt_ch_kernel(Control* c, const BlockDesc* blocks, unsigned long long* maxsig, int nblocks,
                                  double dt) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    c->dt_global = dt;
    c->step = 0;
    c->c_h = ch_from_maxsig(blocks, maxsig, nblocks, dt);
}

// c_h of a step of dt and the psi damping factor the stages take from it
// (e4/fvcell.d:1068-1074, the stage kernels' operations): out[0], out[1].
__global__ void step_ch_damp_kernel(const BlockDesc* blocks, unsigned long long* maxsig, int nblocks, double dt,
                                    double damping_length, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double c_h = ch_from_maxsig(blocks, maxsig, nblocks, dt);
    const double c_h2 = c_h * c_h;
    const double c_p2 = 0.18 * damping_length * c_h;
    out[0] = c_h;
    out[1] = exp(-(c_h2 / c_p2) * dt);
}

}  // namespace gdfv

// ====================================================================== C ABI
using namespace gdfv;

extern "C" {

int gdfv_context_new(void) {
    std::lock_guard<std::mutex> lk(g_mutex);
    int h = g_next++;
    g_ctx[h] = std::make_unique<Context>();
    return h;
}

int gdfv_context_free(int ctx) {
    std::unique_ptr<Context> victim;
    {
        std::lock_guard<std::mutex> lk(g_mutex);
        auto it = g_ctx.find(ctx);
        if (it == g_ctx.end()) return GDFV_ERR_ARG;
        victim = std::move(it->second);
        g_ctx.erase(it);
    }
    if (victim->stream) cudaStreamSynchronize(victim->stream);
    return GDFV_OK;
}

int gdfv_config_set_str(int ctx, const char* key, const char* value) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return fail(c, GDFV_ERR_STATE, "configuration is frozen after gdfv_prepare");
    std::string k = norm(key), v = norm(value);
    if (k == "flux_calculator") {
        if (v == "ausmdv") c->cfg.flux = FLUX_AUSMDV;
        else if (v == "hllc") c->cfg.flux = FLUX_HLLC;
        else if (v == "hlle") c->cfg.flux = FLUX_HLLE;
        else return fail(c, GDFV_ERR_ARG, "unsupported flux_calculator: " + v);
    } else if (k == "gasdynamic_update_scheme") {
        if (v != "predictor_corrector" && v != "pc")
            return fail(c, GDFV_ERR_ARG, "unsupported gasdynamic_update_scheme: " + v);
    } else if (k == "thermo_interpolator") {
        if (v != "rhou") return fail(c, GDFV_ERR_ARG, "unsupported thermo_interpolator: " + v);
    } else if (k == "flux_precision") {
        if (v == "fp64" || v == "double") c->cfg.precision = 0;
        else if (v == "fp32" || v == "float") c->cfg.precision = 1;
        else return fail(c, GDFV_ERR_ARG, "flux_precision is fp64 or fp32");
    } else if (k == "van_albada_variant") {
        if (v == "e4") c->cfg.lmr_epsilon = 0;
        else if (v == "lmr") c->cfg.lmr_epsilon = 1;
        else return fail(c, GDFV_ERR_ARG, "van_albada_variant is e4 or lmr");
    } else {
        return fail(c, GDFV_ERR_ARG, "unknown string option: " + k);
    }
    return GDFV_OK;
}

int gdfv_config_set_int(int ctx, const char* key, long long value) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return fail(c, GDFV_ERR_STATE, "configuration is frozen after gdfv_prepare");
    std::string k = norm(key);
    Config& g = c->cfg;
    int v = (int)value;
    if (k == "interpolation_order") { if (v != 2) return fail(c, GDFV_ERR_ARG, "interpolation_order must be 2"); }
    else if (k == "n_ghost_cell_layers") { if (v != 2) return fail(c, GDFV_ERR_ARG, "n_ghost_cell_layers must be 2"); }
    else if (k == "interpolate_in_local_frame") { if (v != 1) return fail(c, GDFV_ERR_ARG, "interpolate_in_local_frame must be true"); }
    else if (k == "dimensions") g.dims = v;
    else if (k == "MHD" || k == "mhd") g.mhd = v != 0;
    else if (k == "divergence_cleaning") g.divergence_cleaning = v != 0;
    else if (k == "apply_limiter") g.apply_limiter = v != 0;
    else if (k == "extrema_clipping") g.extrema_clipping = v != 0;
    else if (k == "apply_entropy_fix") g.apply_entropy_fix = v != 0;
    else if (k == "glm_reference_indexing") g.glm_reference_indexing = v != 0;
    else if (k == "stringent_cfl") g.stringent_cfl = v != 0;
    else if (k == "cfl_count") { if (v < 1) return fail(c, GDFV_ERR_ARG, "cfl_count >= 1"); g.cfl_count = v; }
    else if (k == "max_attempts_for_step") { if (v < 1) return fail(c, GDFV_ERR_ARG, "max_attempts_for_step >= 1"); g.max_attempts = v; }
    else if (k == "max_invalid_cells") g.max_invalid_cells = v;
    else if (k == "fixed_time_step") g.fixed_time_step = v != 0;
    else if (k == "tile_kchunk") { if (v < 0) return fail(c, GDFV_ERR_ARG, "tile_kchunk >= 0"); g.tile_kchunk = v; }
    else if (k == "persistent") g.persistent = v != 0;
    else if (k == "tile_width") {
        if (v != 16 && v != 32) return fail(c, GDFV_ERR_ARG, "tile_width is 16 or 32");
        g.tile_width = (int)v;
    }
    else if (k == "autotune") g.autotune = v != 0;
    else return fail(c, GDFV_ERR_ARG, "unknown integer option: " + k);
    return GDFV_OK;
}

int gdfv_config_set_double(int ctx, const char* key, double value) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return fail(c, GDFV_ERR_STATE, "configuration is frozen after gdfv_prepare");
    std::string k = norm(key);
    Config& g = c->cfg;
    if (k == "cfl_value") g.cfl_value = value;
    else if (k == "dt_init") g.dt_init = value;
    else if (k == "dt_max") g.dt_max = value;
    else if (k == "epsilon_van_albada") g.eps_van_albada = value;
    else if (k == "r" || k == "R") g.R = value;
    else if (k == "gamma") g.gamma = value;
    else if (k == "divb_damping_length" || k == "divB_damping_length") g.divB_damping_length = value;
    else if (k == "flowstate_limits_max_velocity") g.max_velocity = value;
    else if (k == "flowstate_limits_max_temp") g.max_temp = value;
    else if (k == "flowstate_limits_min_temp") g.min_temp = value;
    else return fail(c, GDFV_ERR_ARG, "unknown real option: " + k);
    return GDFV_OK;
}

int gdfv_config_get_double(int ctx, const char* key, double* value) {
    Context* c = get_ctx(ctx);
    if (!c || !value) return fail(c, GDFV_ERR_ARG, "bad argument");
    std::string k = norm(key);
    Config& g = c->cfg;
    if (k == "cfl_value") *value = g.cfl_value;
    else if (k == "dt_init") *value = g.dt_init;
    else if (k == "dt_max") *value = g.dt_max;
    else if (k == "epsilon_van_albada") *value = g.eps_van_albada;
    else if (k == "R" || k == "r") *value = g.R;
    else if (k == "gamma") *value = g.gamma;
    else if (k == "divB_damping_length" || k == "divb_damping_length") *value = g.divB_damping_length;
    else if (k == "tile_kchunk") *value = g.tile_kchunk;
    else if (k == "persistent") *value = g.persistent;
    else if (k == "tile_width") *value = g.tile_width;
    else if (k == "autotune") *value = g.autotune;
    else if (k == "autotune_stage_ms") *value = c->tune_ms;
    else if (k == "tile_rows") *value = tile_rows(g.precision, g.mhd);
    else if (k == "tile_rows_corrector")   // the float Euler path runs both stages on the first table
        *value = c->n_tiles2 > 0 && !c->prim[0] ? tile_rows_corrector(g.precision, g.mhd) : tile_rows(g.precision, g.mhd);
    else return fail(c, GDFV_ERR_ARG, "unknown real option: " + k);
    return GDFV_OK;
}

int gdfv_block_new(int ctx, int nic, int njc, int nkc, double dx, double dy, double dz, double x0, double y0,
                   double z0) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return fail(c, GDFV_ERR_STATE, "blocks are frozen after gdfv_prepare");
    if (nic < 1 || njc < 1 || nkc < 1 || !(dx > 0) || !(dy > 0) || !(dz > 0))
        return fail(c, GDFV_ERR_ARG, "block sizes and spacings must be positive");
    if ((long long)nic * njc * nkc > (1ll << 34)) return fail(c, GDFV_ERR_ARG, "block too large");
    HostBlock b;
    b.n[0] = nic; b.n[1] = njc; b.n[2] = nkc;
    b.len[0] = dx; b.len[1] = dy; b.len[2] = dz;
    b.origin[0] = x0; b.origin[1] = y0; b.origin[2] = z0;
    c->blocks.push_back(b);
    return (int)c->blocks.size() - 1;
}

int gdfv_block_new_graded(int ctx, int nic, int njc, int nkc, const double* xv, const double* yv, const double* zv) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return fail(c, GDFV_ERR_STATE, "blocks are frozen after gdfv_prepare");
    if (nic < 1 || njc < 1 || nkc < 1 || !xv || !yv || !zv) return fail(c, GDFV_ERR_ARG, "bad block size or vertices");
    if ((long long)nic * njc * nkc > (1ll << 34)) return fail(c, GDFV_ERR_ARG, "block too large");
    HostBlock b;
    b.n[0] = nic; b.n[1] = njc; b.n[2] = nkc;
    const double* v[3] = {xv, yv, zv};
    for (int d = 0; d < 3; ++d) {
        b.vert[d].assign(v[d], v[d] + b.n[d] + 1);
        for (int cc = 0; cc < b.n[d]; ++cc)
            if (!(b.vert[d][cc + 1] - b.vert[d][cc] > 0.0))
                return fail(c, GDFV_ERR_ARG, "vertex coordinates must increase along each axis");
        b.len[d] = b.vert[d][1] - b.vert[d][0];
        b.origin[d] = b.vert[d][0];
    }
    c->blocks.push_back(b);
    return (int)c->blocks.size() - 1;
}

int gdfv_block_set_bc(int ctx, int blk, int face, const char* bc_type, int x_order, int other_blk, int other_face,
                      const double* inflow) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return fail(c, GDFV_ERR_STATE, "boundary conditions are frozen after gdfv_prepare");
    if (blk < 0 || blk >= (int)c->blocks.size() || face < 0 || face > 5) return fail(c, GDFV_ERR_ARG, "bad block or face");
    std::string t = norm(bc_type);
    HostBC bc;
    if (t == "wall_with_slip" || t == "wallbc_withslip" || t == "slip_wall") bc.type = BC_SLIP_WALL;
    else if (t == "outflow_simple_extrapolate" || t == "extrapolate") bc.type = BC_EXTRAPOLATE;
    else if (t == "inflow_supersonic") bc.type = BC_INFLOW;
    else if (t == "exchange_over_full_face" || t == "exchange" || t == "full_face_copy") bc.type = BC_EXCHANGE;
    else if (t == "outflow_fixed_p") bc.type = BC_FIXED_P;
    else if (t == "outflow_fixed_p_and_t") bc.type = BC_FIXED_PT;
    else if (t == "outflow_simple_flux" || t == "outflow_simple") bc.type = BC_SIMPLE_FLUX;
    else return fail(c, GDFV_ERR_ARG, "unsupported boundary condition: " + t);
    bc.x_order = x_order;
    bc.other = other_blk;
    bc.other_face = other_face;
    if (bc.type == BC_INFLOW) {
        if (!inflow) return fail(c, GDFV_ERR_ARG, "inflow_supersonic needs a flow state");
        for (int q = 0; q < 9; ++q) bc.inflow[q] = inflow[q];
    }
    if (bc.type == BC_FIXED_P || bc.type == BC_FIXED_PT) {   // inflow = {p_outside, T_outside}
        if (!inflow || !(inflow[0] > 0.0) || (bc.type == BC_FIXED_PT && !(inflow[1] > 0.0)))
            return fail(c, GDFV_ERR_ARG, "outflow_fixed_p needs p_outside > 0 (and T_outside > 0 with _and_t)");
        bc.inflow[0] = inflow[0];
        bc.inflow[1] = bc.type == BC_FIXED_PT ? inflow[1] : 0.0;
    }
    c->blocks[blk].bc[face] = bc;
    return GDFV_OK;
}

int gdfv_block_set_exchange(int ctx, int blk, int face, int other_blk, int other_face, int orientation,
                            const double* Rmatrix) {
    const int rc = gdfv_block_set_bc(ctx, blk, face, "exchange_over_full_face", 0, other_blk, other_face, nullptr);
    if (rc != GDFV_OK) return rc;
    Context* c = get_ctx(ctx);
    if (orientation < 0 || orientation > 3) return fail(c, GDFV_ERR_ARG, "exchange orientation must be 0..3");
    HostBC& bc = c->blocks[blk].bc[face];
    bc.orientation = orientation;
    if (Rmatrix) {
        for (int m = 0; m < 9; ++m)
            if (!std::isfinite(Rmatrix[m])) return fail(c, GDFV_ERR_ARG, "Rmatrix entries must be finite");
        bc.rotate = 1;
        for (int m = 0; m < 9; ++m) bc.rot[m] = Rmatrix[m];
    }
    return GDFV_OK;
}

int gdfv_exchange_source(int dims, int face, int other_face, int orientation, const int* n_this, const int* n_other,
                         const int* ijk, int* src) {
    const int nf = dims == 3 ? 6 : 4;
    if ((dims != 2 && dims != 3) || face < 0 || face >= nf || other_face < 0 || other_face >= nf || orientation < 0 ||
        orientation > 3 || !n_this || !n_other || !ijk || !src)
        return fail(nullptr, GDFV_ERR_ARG, "gdfv_exchange_source: bad dims, face, orientation or pointer");
    const int ax = face / 2;
    const int depth = (face & 1) ? ijk[ax] - n_this[ax] : -1 - ijk[ax];
    for (int d = 0; d < 3; ++d)
        if (d != ax && (ijk[d] < 0 || ijk[d] >= n_this[d]))
            return fail(nullptr, GDFV_ERR_ARG, "gdfv_exchange_source: ghost cell not beside the face");
    if (depth < 0 || depth > 1) return fail(nullptr, GDFV_ERR_ARG, "gdfv_exchange_source: ghost depth must be 0 or 1");
    const int xm = exchange_map(dims, face, other_face, orientation);
    for (int d = 0; d < 3; ++d) {
        const int sel = (xm >> (3 * d)) & 3;
        const int v = sel == 3 ? depth : ijk[sel];
        src[d] = ((xm >> (3 * d + 2)) & 1) ? n_other[d] - 1 - v : v;
        if (src[d] < 0 || src[d] >= n_other[d])
            return fail(nullptr, GDFV_ERR_ARG, "gdfv_exchange_source: the faces differ in size under this map");
    }
    return GDFV_OK;
}

int gdfv_prepare(int ctx) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->prepared) return GDFV_OK;
    return do_prepare(c);
}

long long gdfv_block_ncells(int ctx, int blk) {
    Context* c = get_ctx(ctx);
    if (!c || blk < 0 || blk >= (int)c->blocks.size()) return -1;
    const HostBlock& b = c->blocks[blk];
    return (long long)b.n[0] * b.n[1] * b.n[2];
}

long long gdfv_total_cells(int ctx) {
    Context* c = get_ctx(ctx);
    if (!c) return -1;
    long long t = 0;
    for (auto& b : c->blocks) t += (long long)b.n[0] * b.n[1] * b.n[2];
    return t;
}

static int check_ready(Context* c, int blk) {
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (!c->prepared) return fail(c, GDFV_ERR_STATE, "call gdfv_prepare first");
    if (blk < -1 || blk >= (int)c->blocks.size()) return fail(c, GDFV_ERR_ARG, "bad block");
    return GDFV_OK;
}

int gdfv_block_set_flow_rhoT(int ctx, int blk, const double* prim) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, blk);
    if (st) return st;
    if (!prim || blk < 0) return fail(c, GDFV_ERR_ARG, "bad argument");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    const HostBlock& b = c->blocks[blk];
    long long n = (long long)b.n[0] * b.n[1] * b.n[2];
    double* d_prim = nullptr;
    CK(cudaMalloc(&d_prim, sizeof(double) * 9 * n));
    cudaError_t e = cudaMemcpyAsync(d_prim, prim, sizeof(double) * 9 * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_bad, 0, sizeof(int), c->stream);
    if (e == cudaSuccess) {
        encode_rhoT_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
            d_prim, n, c->U[c->h_ctl->step & 1], c->total, b.offset, c->P, c->d_bad);
        e = cudaGetLastError();
    }
    int bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, c->d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_prim);
    if (e != cudaSuccess) return cuda_fail(c, e, "set_flow_rhoT");
    if (bad) return fail(c, GDFV_ERR_ARG, "initial state has T <= 0 or rho <= 0");
    c->signal_valid = false;
    c->prims_valid = false;
    return GDFV_OK;
}

int gdfv_block_set_conserved(int ctx, int blk, const double* U) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, blk);
    if (st) return st;
    if (!U || blk < 0) return fail(c, GDFV_ERR_ARG, "bad argument");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    const HostBlock& b = c->blocks[blk];
    long long n = (long long)b.n[0] * b.n[1] * b.n[2];
    double* dst = c->U[c->h_ctl->step & 1];
    for (int q = 0; q < c->nq; ++q)
        CK(cudaMemcpyAsync(dst + q * c->total + b.offset, U + q * n, sizeof(double) * n, cudaMemcpyHostToDevice,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->signal_valid = false;
    c->prims_valid = false;
    return GDFV_OK;
}

int gdfv_block_get_conserved(int ctx, int blk, double* U) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, blk);
    if (st) return st;
    if (!U || blk < 0) return fail(c, GDFV_ERR_ARG, "bad argument");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    const HostBlock& b = c->blocks[blk];
    long long n = (long long)b.n[0] * b.n[1] * b.n[2];
    const double* src = c->U[c->h_ctl->step & 1];
    for (int q = 0; q < c->nq; ++q)
        CK(cudaMemcpyAsync(U + q * n, src + q * c->total + b.offset, sizeof(double) * n, cudaMemcpyDeviceToHost,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return GDFV_OK;
}

int gdfv_block_get_flow(int ctx, int blk, double* out) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, blk);
    if (st) return st;
    if (!out || blk < 0) return fail(c, GDFV_ERR_ARG, "bad argument");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    const HostBlock& b = c->blocks[blk];
    long long n = (long long)b.n[0] * b.n[1] * b.n[2];
    double* d_out = nullptr;
    CK(cudaMalloc(&d_out, sizeof(double) * 12 * n));
    decode_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->U[c->h_ctl->step & 1], c->total, b.offset,
                                                                       n, c->P, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, sizeof(double) * 12 * n, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_out);
    if (e != cudaSuccess) return cuda_fail(c, e, "get_flow");
    return GDFV_OK;
}

}  // extern "C"

namespace gdfv {

// Scratch control record of the fixed-dt step chains, and the current c_h (host read).
int steps_dt_prepare(int ctx) {
    Context* c = get_ctx(ctx);
    if (!c) return GDFV_ERR_ARG;
    if (step_scratch(c)) return GDFV_ERR_CUDA;
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    return GDFV_OK;
}

// Enqueues n fixed-dt steps on `stream`: step m takes dts[m] from the previous output
// (U_in for m = 0) to U_out[m]; U1_out[m] (optional) receives the predictor state.
// fresh: reset the chain's failure counters (otherwise they accumulate over chains).
// steps_dt_prepare must have run.  Uses the context's dU0 and scratch control record,
// so at most one chain may be in flight per context.
cudaError_t enqueue_steps_dt(int ctx, cudaStream_t stream, const double* U_in, double* const* U_out,
                             double* const* U1_out, const double* dts, int n, bool fresh) {
    Context* c = get_ctx(ctx);
    if (!c || !c->step_ctl || !U_in || !U_out || !dts || n < 1) return cudaErrorInvalidValue;
    for (int m = 0; m < n; ++m) {
        const double* src = m == 0 ? U_in : U_out[m - 1];
        // only the last step may omit its output (then only its predictor state is formed)
        if ((!U_out[m] && m < n - 1) || U_out[m] == src || !(dts[m] > 0.0)) return cudaErrorInvalidValue;
    }
    StageArgs A = stage_args(c);
    A.ctl = c->step_ctl;
    A.max_signal = c->step_maxsig;
    A.last_signal = c->step_lastsig;
    const bool ch_rule = c->cfg.mhd && c->P.divergence_cleaning;
    for (int m = 0; m < n; ++m) {
        const double* src = m == 0 ? U_in : U_out[m - 1];
        A.Ubuf[0] = const_cast<double*>(src);
        A.Ubuf[1] = U_out[m];
        A.R_out = U1_out ? U1_out[m] : nullptr;   // the predictor stage writes U1 there
        if (m == 0 && fresh)
            step_dt_begin_kernel<<<1, 256, 0, stream>>>(c->step_ctl, c->step_maxsig, (int)c->blocks.size(), dts[0],
                                                        c->h_ctl->c_h);
        else if (!ch_rule)
            step_dt_next_kernel<<<1, 1, 0, stream>>>(c->step_ctl, dts[m]);
        cudaError_t e = cudaGetLastError();
        if (ch_rule) {
            // the step's c_h from the signal maxima of its start state, as gdfv_run forms
            // it: a scan of the chain's input, then the maxima each corrector leaves
            if (e == cudaSuccess && m == 0)
                e = enqueue_signal_scan(c, stream, src, c->step_maxsig, c->step_lastsig, c->ch_bad);
            if (e == cudaSuccess) {
                step_dt_ch_kernel<<<1, 1, 0, stream>>>(c->step_ctl, c->d_blocks, c->step_maxsig, (int)c->blocks.size(),
                                                       dts[m]);
                e = cudaGetLastError();
            }
        }
        if (e == cudaSuccess) e = c->cfg.precision == 0 ? launch_stage_fp64(1, c->cfg.flux, c->cfg.mhd, A, stream)
                                                        : launch_stage_fp32(1, c->cfg.flux, c->cfg.mhd, A, stream);
        A.R_out = nullptr;
        if (e == cudaSuccess && U_out[m])
            e = c->cfg.precision == 0 ? launch_stage_fp64(2, c->cfg.flux, c->cfg.mhd, A, stream)
                                      : launch_stage_fp32(2, c->cfg.flux, c->cfg.mhd, A, stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The c_h of a step of dt that starts at U and the psi damping factor of its stages
// (out[0], out[1], device), as gdfv_run forms them, enqueued on `stream` with the
// context's adjoint scan scratch (steps_dt_prepare must have run).
cudaError_t enqueue_step_ch(int ctx, cudaStream_t stream, const double* U, double dt, double* out) {
    Context* c = get_ctx(ctx);
    if (!c || !c->ch_maxsig || !U || !out) return cudaErrorInvalidValue;
    cudaError_t e = enqueue_signal_scan(c, stream, U, c->ch_maxsig, c->ch_lastsig, c->ch_bad);
    if (e != cudaSuccess) return e;
    step_ch_damp_kernel<<<1, 1, 0, stream>>>(c->d_blocks, c->ch_maxsig, (int)c->blocks.size(), dt,
                                            c->cfg.divB_damping_length, out);
    return cudaGetLastError();
}

// Waits for `stream` and reports the failure counters of the chains run since the
// last fresh start: 0, GDFV_ERR_STEP_FAILED or GDFV_ERR_BAD_CELLS (with the message).
int steps_dt_status(int ctx, cudaStream_t stream) {
    Context* c = get_ctx(ctx);
    if (!c) return GDFV_ERR_ARG;
    Control h{};
    CK(cudaMemcpyAsync(&h, c->step_ctl, sizeof(Control), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (h.n_fail > 0)
        return fail(c, GDFV_ERR_STEP_FAILED, "fixed-dt step: a cell failed to decode." + bad_cell_text(c, h.first_bad_cell));
    if (h.n_invalid1 > c->cfg.max_invalid_cells || h.n_invalid2 > c->cfg.max_invalid_cells)
        return fail(c, GDFV_ERR_BAD_CELLS, "fixed-dt step: too many bad cells." + bad_cell_text(c, h.first_bad_cell));
    return GDFV_OK;
}

// The context's extra streams (created on first use): which = 0 at the lowest
// priority, 1 at the highest.
cudaStream_t context_aux_stream(int ctx, int which) {
    Context* c = get_ctx(ctx);
    if (!c || which < 0 || which > 1) return nullptr;
    if (!c->aux_stream[which]) {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) return nullptr;
        if (cudaStreamCreateWithPriority(&c->aux_stream[which], cudaStreamNonBlocking, which ? greatest : least) !=
            cudaSuccess)
            c->aux_stream[which] = nullptr;
    }
    return c->aux_stream[which];
}

int upload_tiles(Context* c, const std::vector<TileDesc>& tiles, int n1, int n2, int n3, int n4) {
    CK(cudaStreamSynchronize(c->stream));
    if (tiles.size() > c->tiles_cap) {
        if (c->d_tiles) cudaFree(c->d_tiles);
        c->d_tiles = nullptr;
        c->tiles_cap = 0;
        CK(cudaMalloc(&c->d_tiles, sizeof(TileDesc) * tiles.size()));
        c->tiles_cap = tiles.size();
    }
    CK(cudaMemcpy(c->d_tiles, tiles.data(), sizeof(TileDesc) * tiles.size(), cudaMemcpyHostToDevice));
    c->n_tiles = n1;
    c->n_tiles2 = n2;
    c->n_prim_wide = n3;
    c->n_prim_narrow = n4;
    drop_graphs(c);  // captured the old table
    return GDFV_OK;
}

// Autotuner: for each tile k-chunk and launch form (persistent grid or one CTA
// per tile) -- and for the kernel on decoded primitives, both tile widths -- time
// stage 1 + stage 2 on the current state and keep the fastest.
// The trial steps use a scratch control record with dt = 0 and write only the
// idle state buffer and dU0, so the solution is not changed.
int autotune(Context* c) {
    if (step_scratch(c)) return GDFV_ERR_CUDA;
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    const int parity = c->h_ctl->step & 1;
    const double c_h = c->h_ctl->c_h > 0.0 ? c->h_ctl->c_h : 1.0;
    int maxk = 1;
    for (const HostBlock& hb : c->blocks) maxk = std::max(maxk, hb.n[2]);
    std::vector<int> kcs;
    if (c->cfg.dims == 2) kcs.push_back(1);
    else
        for (int kc : {8, 12, 16, 24, 32, 64, 128})
            if (kc <= maxk || kcs.empty()) kcs.push_back(kc);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best = 1e30;
    int best_kc = c->cfg.tile_kchunk, best_p = c->cfg.persistent, best_w = c->cfg.tile_width;
    // tile widths of the kernel on decoded primitives
    std::vector<int> widths = {c->cfg.tile_width};
    if (c->prim[0]) widths = {32, 16};
    std::vector<TileDesc> tiles;
    cudaError_t e = cudaSuccess;
    const int reps = 3;
    for (int tw : widths)
    for (int kc : kcs) {
        c->cfg.tile_width = tw;
        int n1 = 0, n2 = 0, n3 = 0, n4 = 0;
        build_tiles(c, kc, tiles, n1, n2, n3, n4);
        int st = upload_tiles(c, tiles, n1, n2, n3, n4);
        if (st) { cudaEventDestroy(e0); cudaEventDestroy(e1); return st; }
        for (int pers = 1; pers >= 0 && e == cudaSuccess; --pers) {
            StageArgs A = stage_args_run(c, parity);
            A.Ubuf[0] = c->U[parity];
            A.Ubuf[1] = c->U[parity ^ 1];
            A.ctl = c->step_ctl;
            A.max_signal = c->step_maxsig;
            A.last_signal = c->step_lastsig;
            A.persistent = pers;
            step_dt_begin_kernel<<<1, 256, 0, c->stream>>>(c->step_ctl, c->step_maxsig, (int)c->blocks.size(), 0.0, c_h);
            e = cudaGetLastError();
            for (int r = -1; r < reps && e == cudaSuccess; ++r) {
                if (r == 0) e = cudaEventRecord(e0, c->stream);
                if (e == cudaSuccess) e = launch_stage(c, 1, A);
                if (e == cudaSuccess) e = launch_stage(c, 2, A);
            }
            if (e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && ms / reps < best) { best = ms / reps; best_kc = kc; best_p = pers; best_w = tw; }
        }
        if (e != cudaSuccess) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(c, e, "autotune");
    c->cfg.tile_kchunk = best_kc;
    c->cfg.persistent = best_p;
    c->cfg.tile_width = best_w;
    int n1 = 0, n2 = 0, n3 = 0, n4 = 0;
    build_tiles(c, best_kc, tiles, n1, n2, n3, n4);
    int st = upload_tiles(c, tiles, n1, n2, n3, n4);
    if (st) return st;
    c->tuned = true;
    c->tune_ms = best;
    return GDFV_OK;
}

}  // namespace gdfv

extern "C" {

int gdfv_run(int ctx, int max_steps, double max_time, int* steps_taken) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (steps_taken) *steps_taken = 0;
    if (max_steps <= 0) return GDFV_OK;
    if (!c->signal_valid) {
        if ((st = scan_signal(c)) != GDFV_OK) return st;
    }
    if ((st = ensure_prims(c)) != GDFV_OK) return st;
    if (c->cfg.autotune && !c->tuned) {
        if ((st = autotune(c)) != GDFV_OK) return st;
    }
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    if (c->h_ctl->status != ST_OK) return fail(c, GDFV_ERR_STATE, "a previous run failed; reset the state");
    const int start_step = c->h_ctl->step;
    c->h_ctl->step_limit = start_step + max_steps;
    c->h_ctl->max_time = max_time;
    c->h_ctl->halted = 0;
    c->h_ctl->steps_done = 0;
    if (write_ctl(c)) return GDFV_ERR_CUDA;
    if (!c->graph) {
        if ((st = build_graph(c)) != GDFV_OK) return st;
    }
    // Replay the captured steps in batches sized to what is left, reading the
    // control record back after each batch.  Steps past the halt are no-ops.
    const long long slot_budget = (long long)(c->cfg.max_attempts + 1) * (max_steps + 1) + 2 * c->graph_steps;
    long long launched = 0;
    while (!c->h_ctl->halted && c->h_ctl->status == ST_OK && launched < slot_budget) {
        long long remaining = (long long)c->h_ctl->step_limit - c->h_ctl->step;
        if (max_time > 0.0 && c->h_ctl->dt_global > 0.0) {
            double est = std::ceil((max_time - c->h_ctl->time) / c->h_ctl->dt_global) + 1.0;
            if (est < (double)remaining) remaining = (long long)std::max(1.0, est);
        }
        if (c->h_ctl->retrying) remaining += 1;
        // whole batches, then single slots for the rest
        remaining = std::max<long long>(1, remaining);
        const int graphs = (int)std::min<long long>(64, remaining / c->graph_steps);
        const int singles = graphs < 64 ? (int)(remaining % c->graph_steps) : 0;
        for (int g = 0; g < graphs; ++g) CK(cudaGraphLaunch(c->graph, c->stream));
        for (int g = 0; g < singles; ++g) CK(cudaGraphLaunch(c->graph1, c->stream));
        launched += (long long)graphs * c->graph_steps + singles;
        if (read_ctl(c)) return GDFV_ERR_CUDA;
    }
    if (steps_taken) *steps_taken = c->h_ctl->step - start_step;
    if (c->h_ctl->status == ST_TOO_MANY_BAD_CELLS)
        return fail(c, GDFV_ERR_BAD_CELLS, "Too many bad cells during explicit gasdynamic update." +
                                               bad_cell_text(c, c->h_ctl->first_bad_cell));
    if (c->h_ctl->status == ST_DECODE_FAILED)
        return fail(c, GDFV_ERR_STEP_FAILED, "Explicit update failed after max_attempts_for_step attempts." +
                                                 bad_cell_text(c, c->h_ctl->first_bad_cell));
    return GDFV_OK;
}

int gdfv_run_record(int ctx, int nsteps, double* const* states_dev, double* const* preds_dev, double* dts) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (nsteps < 1 || !states_dev || !preds_dev || !dts)
        return fail(c, GDFV_ERR_ARG, "gdfv_run_record needs nsteps >= 1, the two pointer arrays and dts");
    if (!c->signal_valid) {
        if ((st = scan_signal(c)) != GDFV_OK) return st;
    }
    if ((st = ensure_prims(c)) != GDFV_OK) return st;
    if (c->cfg.autotune && !c->tuned) {
        if ((st = autotune(c)) != GDFV_OK) return st;
    }
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    if (c->h_ctl->status != ST_OK) return fail(c, GDFV_ERR_STATE, "a previous run failed; reset the state");
    const int start_step = c->h_ctl->step;
    c->h_ctl->step_limit = start_step + nsteps;
    c->h_ctl->max_time = 0.0;
    c->h_ctl->halted = 0;
    c->h_ctl->steps_done = 0;
    if (write_ctl(c)) return GDFV_ERR_CUDA;
    if (!c->graph) {
        if ((st = build_graph(c)) != GDFV_OK) return st;
    }
    if (c->rec_cap < nsteps) {
        if (c->d_rec) cudaFree(c->d_rec);
        c->d_rec = nullptr;
        c->rec_cap = 0;
        CK(cudaMalloc(&c->d_rec, sizeof(double) * ((size_t)nsteps + 1)));
        c->rec_cap = nsteps;
    }
    int* flag = reinterpret_cast<int*>(c->d_rec + nsteps);
    CK(cudaMemsetAsync(flag, 0, sizeof(int), c->stream));
    const long long n = (long long)c->nq * c->total;
    const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 8LL * 148);
    // one step slot per step, each followed by its record: no host round trip in between
    for (int m = 0; m < nsteps; ++m) {
        CK(cudaGraphLaunch(c->graph1, c->stream));
        record_step_kernel<<<grid, 256, 0, c->stream>>>(c->d_ctl, c->U[0], c->U[1], c->dU0, n, start_step + m + 1,
                                                        states_dev[m], preds_dev[m], c->d_rec + m, flag);
        CK(cudaGetLastError());
    }
    int h_flag = 0;
    CK(cudaMemcpyAsync(&h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(dts, c->d_rec, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, c->stream));
    if (read_ctl(c)) return GDFV_ERR_CUDA;   // synchronises the stream
    if (c->h_ctl->status == ST_TOO_MANY_BAD_CELLS)
        return fail(c, GDFV_ERR_BAD_CELLS, "Too many bad cells during explicit gasdynamic update." +
                                               bad_cell_text(c, c->h_ctl->first_bad_cell));
    if (c->h_ctl->status == ST_DECODE_FAILED)
        return fail(c, GDFV_ERR_STEP_FAILED, "Explicit update failed after max_attempts_for_step attempts." +
                                                 bad_cell_text(c, c->h_ctl->first_bad_cell));
    if (h_flag || c->h_ctl->step != start_step + nsteps)
        return fail(c, GDFV_ERR_STATE, "gdfv_run_record: a step was retried, so the record is incomplete (the "
                                       "state has moved on; take the steps with gdfv_run instead)");
    return GDFV_OK;
}

int gdfv_last_bad_cell(int ctx, int* blk, int* ijk, double* pos) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (c->last_bad_cell < 0) return fail(c, GDFV_ERR_STATE, "no failed step has reported a cell");
    locate_cell(c, c->last_bad_cell, blk, ijk, pos);
    return GDFV_OK;
}

int gdfv_set_inflow(int ctx, int index, const double* state) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (index < 0 || index >= c->n_inflow || !state) return fail(c, GDFV_ERR_ARG, "bad inflow index or state");
    const Config& g = c->cfg;
    const double p = state[0], T = state[1];
    if (!(p > 0.0) || !(T > 0.0)) return fail(c, GDFV_ERR_ARG, "inflow needs p > 0 and T > 0");
    // as gdfv_prepare builds it: FlowState:new{p=, T=} (update_thermo_from_pT, update_sound_speed)
    InflowState s{};
    s.p = p;
    s.rho = p / (T * g.R);
    s.u = (g.R / (g.gamma - 1.0)) * T;
    s.a = std::sqrt(g.gamma * g.R * T);
    for (int d = 0; d < 3; ++d) { s.vel[d] = state[2 + d]; s.B[d] = state[5 + d]; }
    s.psi = state[8];
    CK(cudaMemcpyAsync(c->d_inflow + index, &s, sizeof(InflowState), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::copy(state, state + 9, c->h_inflow.begin() + 9 * (size_t)index);
    return GDFV_OK;
}

int gdfv_get_time(int ctx, double* out5, int* step) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    if (out5) {
        out5[0] = c->h_ctl->time; out5[1] = c->h_ctl->dt_global; out5[2] = c->h_ctl->c_h;
        out5[3] = c->h_ctl->cfl_max; out5[4] = c->h_ctl->dt_allow;
    }
    if (step) *step = c->h_ctl->step;
    return GDFV_OK;
}

int gdfv_set_time(int ctx, double time, int step, double dt_global) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (step < 0 || !(dt_global > 0)) return fail(c, GDFV_ERR_ARG, "bad time state");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    int old_parity = c->h_ctl->step & 1;
    if ((step & 1) != old_parity) {
        CK(cudaMemcpyAsync(c->U[step & 1], c->U[old_parity], sizeof(double) * c->nq * c->total,
                           cudaMemcpyDeviceToDevice, c->stream));
    }
    c->h_ctl->time = time;
    c->h_ctl->step = step;
    c->h_ctl->dt_global = dt_global;
    c->h_ctl->status = ST_OK;
    c->h_ctl->halted = 0;
    c->h_ctl->attempt = 0;
    c->h_ctl->retrying = 0;
    if (write_ctl(c)) return GDFV_ERR_CUDA;
    c->signal_valid = false;
    c->prims_valid = false;
    return GDFV_OK;
}

int gdfv_residual(int ctx, const double* U_dev, double* R_dev) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (!U_dev || !R_dev) return fail(c, GDFV_ERR_ARG, "null pointer");
    StageArgs A = stage_args(c);
    A.U_in = U_dev;
    A.R_out = R_dev;
    CK(launch_stage(c, 0, A));
    CK(cudaStreamSynchronize(c->stream));
    return GDFV_OK;
}

int gdfv_residual_jvp(int ctx, const double* U_dev, const double* v_dev, const double* R0_dev, double sigma,
                      double* Jv_dev, double* sigma_used) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (!U_dev || !v_dev || !Jv_dev) return fail(c, GDFV_ERR_ARG, "null pointer");
    const long long n = (long long)c->nq * c->total;
    if (!c->jvp_scratch) CK(cudaMalloc(&c->jvp_scratch, sizeof(double) * (3 * n + 2 * kJvpSumBlocks)));
    double* Up = c->jvp_scratch;
    double* R0 = Up + n;
    double* R1 = R0 + n;
    double* partial = R1 + n;
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (!(sigma > 0.0)) {
        // Knoll-McHugh perturbation (e4/steadystate_core.d:3040-3078):
        // sigma = sum(eps |U| + eps) / (N max(||v||, sqrt(eps))), eps = 1e-7
        const double eps = 1.0e-07;
        jvp_sums_kernel<<<kJvpSumBlocks, 256, 0, c->stream>>>(U_dev, v_dev, n, eps, partial);
        CK(cudaGetLastError());
        std::vector<double> h(2 * kJvpSumBlocks);
        CK(cudaMemcpyAsync(h.data(), partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        double sum = 0.0, v2 = 0.0;
        for (int b = 0; b < kJvpSumBlocks; ++b) { sum += h[2 * b]; v2 += h[2 * b + 1]; }
        double vnorm = std::sqrt(v2);
        if (vnorm < std::sqrt(eps)) vnorm = std::sqrt(eps);
        sigma = sum / ((double)n * vnorm);
    }
    if (sigma_used) *sigma_used = sigma;
    StageArgs A = stage_args(c);
    if (!R0_dev) {
        A.U_in = U_dev;
        A.R_out = R0;
        CK(launch_stage(c, 0, A));
        R0_dev = R0;
    }
    jvp_axpy_kernel<<<nb, 256, 0, c->stream>>>(U_dev, v_dev, sigma, n, Up);
    CK(cudaGetLastError());
    A.U_in = Up;
    A.R_out = R1;
    CK(launch_stage(c, 0, A));
    jvp_diff_kernel<<<nb, 256, 0, c->stream>>>(R1, R0_dev, sigma, n, Jv_dev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return GDFV_OK;
}

int gdfv_step_dt(int ctx, const double* U_in_dev, double* U_out_dev, double dt, double* U1_out_dev) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (!U_in_dev || !U_out_dev || U_in_dev == U_out_dev || !(dt > 0.0))
        return fail(c, GDFV_ERR_ARG, "gdfv_step_dt needs distinct input/output arrays and dt > 0");
    if (step_scratch(c)) return GDFV_ERR_CUDA;
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    StageArgs A = stage_args(c);
    A.Ubuf[0] = const_cast<double*>(U_in_dev);
    A.Ubuf[1] = U_out_dev;
    A.ctl = c->step_ctl;
    A.max_signal = c->step_maxsig;
    A.last_signal = c->step_lastsig;
    step_dt_begin_kernel<<<1, 256, 0, c->stream>>>(c->step_ctl, c->step_maxsig, (int)c->blocks.size(), dt,
                                                   c->h_ctl->c_h);
    CK(cudaGetLastError());
    if (c->cfg.mhd && c->P.divergence_cleaning) {   // c_h of U_in, as gdfv_run forms it
        CK(enqueue_signal_scan(c, c->stream, U_in_dev, c->step_maxsig, c->step_lastsig, c->ch_bad));
        step_dt_ch_kernel<<<1, 1, 0, c->stream>>>(c->step_ctl, c->d_blocks, c->step_maxsig, (int)c->blocks.size(), dt);
        CK(cudaGetLastError());
    }
    CK(launch_stage(c, 1, A));
    if (U1_out_dev) {
        long long n = (long long)c->nq * c->total;
        predictor_state_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(U_in_dev, c->dU0, dt, n, U1_out_dev);
        CK(cudaGetLastError());
    }
    CK(launch_stage(c, 2, A));
    Control h{};
    CK(cudaMemcpyAsync(&h, c->step_ctl, sizeof(Control), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (h.n_fail > 0)
        return fail(c, GDFV_ERR_STEP_FAILED, "gdfv_step_dt: a cell failed to decode." + bad_cell_text(c, h.first_bad_cell));
    if (h.n_invalid1 > c->cfg.max_invalid_cells || h.n_invalid2 > c->cfg.max_invalid_cells)
        return fail(c, GDFV_ERR_BAD_CELLS, "gdfv_step_dt: too many bad cells." + bad_cell_text(c, h.first_bad_cell));
    return GDFV_OK;
}

int gdfv_steps_dt(int ctx, const double* U_in_dev, double* const* U_out_dev, double* const* U1_out_dev,
                  const double* dts, int n) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if ((st = steps_dt_prepare(ctx))) return st;
    cudaError_t e = enqueue_steps_dt(ctx, c->stream, U_in_dev, U_out_dev, U1_out_dev, dts, n, true);
    if (e == cudaErrorInvalidValue) return fail(c, GDFV_ERR_ARG, "gdfv_steps_dt needs U_in, n >= 1 distinct output arrays and dt > 0");
    if (e != cudaSuccess) return cuda_fail(c, e, "gdfv_steps_dt");
    return steps_dt_status(ctx, c->stream);
}

int gdfv_last_predictor_state(int ctx, const double* U0_dev, double* U1_out_dev) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (!U0_dev || !U1_out_dev || U0_dev == U1_out_dev)
        return fail(c, GDFV_ERR_ARG, "gdfv_last_predictor_state needs distinct U0 and U1 arrays");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    if (c->h_ctl->step < 1) return fail(c, GDFV_ERR_STATE, "no step taken yet");
    const long long n = (long long)c->nq * c->total;
    predictor_state_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(U0_dev, c->dU0, c->h_ctl->dt_global, n,
                                                                               U1_out_dev);
    CK(cudaGetLastError());
    return GDFV_OK;
}

int gdfv_residual_norms(int ctx, double* Linf, double* L2) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (!L2) return fail(c, GDFV_ERR_ARG, "null pointer");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    if (c->h_ctl->step < 1) return fail(c, GDFV_ERR_STATE, "no step taken yet");
    int n_sm = 0, per_sm = 0;
    CK(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, c->device));
    const int nq = c->nq;
    // one wave of resident CTAs (at most 8 per SM: the partials' capacity)
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, nq == 10 ? residual_norms_kernel<10> : residual_norms_kernel<5>, kNormThreads, 0));
    const long long want = (c->total + kNormThreads - 1) / kNormThreads;
    const int ncta = (int)std::max(1LL, std::min<long long>(want, (long long)std::min(std::max(per_sm, 1), 8) * n_sm));
    if (!c->norm_scratch) CK(cudaMalloc(&c->norm_scratch, sizeof(double) * ((size_t)8 * n_sm * 11 + 16)));
    double* out = c->norm_scratch;
    double* partial = c->norm_scratch + 16;
    if (nq == 10)
        residual_norms_kernel<10><<<ncta, kNormThreads, 0, c->stream>>>(c->dU0, c->total, c->cfg.dims == 3, partial);
    else
        residual_norms_kernel<5><<<ncta, kNormThreads, 0, c->stream>>>(c->dU0, c->total, c->cfg.dims == 3, partial);
    CK(cudaGetLastError());
    residual_norms_final_kernel<<<1, 32 * (nq + 1), 0, c->stream>>>(partial, ncta, nq, out);
    CK(cudaGetLastError());
    double h[11];
    CK(cudaMemcpyAsync(h, out, sizeof(double) * (nq + 1), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (Linf)
        for (int q = 0; q < nq; ++q) Linf[q] = h[q];
    *L2 = h[nq];
    return GDFV_OK;
}

int gdfv_state_device_ptr(int ctx, double** U_dev) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (!U_dev) return fail(c, GDFV_ERR_ARG, "null pointer");
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    *U_dev = c->U[c->h_ctl->step & 1];
    c->prims_valid = false;   // the caller may write the state through the pointer
    return GDFV_OK;
}

int gdfv_set_stream(int ctx, void* stream) {
    Context* c = get_ctx(ctx);
    if (!c) return fail(nullptr, GDFV_ERR_ARG, "bad context");
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    drop_graphs(c);
    return GDFV_OK;
}

int gdfv_time_stages(int ctx, int reps, double* ms) {
    Context* c = get_ctx(ctx);
    int st = check_ready(c, -1);
    if (st) return st;
    if (reps < 1 || !ms) return fail(c, GDFV_ERR_ARG, "bad argument");
    if (!c->signal_valid && (st = scan_signal(c)) != GDFV_OK) return st;
    if ((st = ensure_prims(c)) != GDFV_OK) return st;
    if (read_ctl(c)) return GDFV_ERR_CUDA;
    Control saved = *c->h_ctl;
    // a step that cannot halt: the kernels run, the step counter does not move
    c->h_ctl->step_limit = INT_MAX;
    c->h_ctl->max_time = 0.0;
    c->h_ctl->halted = 0;
    c->h_ctl->n_fail = 0;
    c->h_ctl->n_invalid1 = 0;
    if (write_ctl(c)) return GDFV_ERR_CUDA;
    StageArgs A = stage_args_run(c);
    cudaEvent_t e0, e1, e2;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventCreate(&e2));
    float t1 = 0, t2 = 0;
    for (int r = 0; r < reps + 1; ++r) {
        CK(cudaEventRecord(e0, c->stream));
        CK(launch_stage(c, 1, A));
        CK(cudaEventRecord(e1, c->stream));
        CK(launch_stage(c, 2, A));
        CK(cudaEventRecord(e2, c->stream));
        CK(cudaEventSynchronize(e2));
        float a = 0, b = 0;
        CK(cudaEventElapsedTime(&a, e0, e1));
        CK(cudaEventElapsedTime(&b, e1, e2));
        if (r > 0) { t1 += a; t2 += b; }  // first repetition is a warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    ms[0] = t1 / reps;
    ms[1] = t2 / reps;
    // stage 2 wrote the other buffer; the current state and the controller are untouched
    *c->h_ctl = saved;
    if (write_ctl(c)) return GDFV_ERR_CUDA;
    c->signal_valid = false;  // the timed corrector stages overwrote the signal maxima
    return GDFV_OK;
}

int gdfv_last_error(int ctx, char* buf, int n) {
    if (!buf || n <= 0) return GDFV_ERR_ARG;
    Context* c = get_ctx(ctx);
    std::snprintf(buf, (size_t)n, "%s", c ? c->err.c_str() : g_err.c_str());
    return GDFV_OK;
}

}  // extern "C"
