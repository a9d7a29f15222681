/* gdfv.h -- C ABI of the B200 structured-grid finite-volume library (libgdfv.so).
 *
 * Drop-in boundary for the explicit structured-grid update that Eilmer-4 and
 * chicken share.  Conventions follow the reference's loadable-library wrappers
 * (src/gas/gas_cwrap.d): integer handles, plain pointers and sizes, status 0 on
 * success and a negative value on error, never an exception across the ABI;
 * the message of the last error is kept per context (gdfv_last_error).
 *
 * Arrays are structure-of-arrays, FP64, cell index i fastest:
 *   conserved  [nq][ncells]  nq = 5 (mass, x/y/z-momentum, total energy) or 10 with MHD
 *              (+ xB, yB, zB, psi, divB), e4/conservedquantities.d:148-197
 *   flow       [12][ncells]  rho, vel.x, vel.y, vel.z, u, p, T, a, B.x, B.y, B.z, psi
 *   rhoT state [9][ncells]   rho, vel.x, vel.y, vel.z, T, B.x, B.y, B.z, psi
 * "Host" arguments are host memory; "device" arguments are device memory on the
 * context's GPU (for example torch's data_ptr()).
 */
#ifndef GDFV_H
#define GDFV_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define GDFV_OK 0
#define GDFV_ERR_ARG (-1)          /* bad handle, key, value or size */
#define GDFV_ERR_BAD_CELLS (-2)    /* too many invalid cells: the run stopped */
#define GDFV_ERR_STEP_FAILED (-3)  /* decode failed on every attempt of a step */
#define GDFV_ERR_CUDA (-4)         /* a CUDA call failed */
#define GDFV_ERR_STATE (-5)        /* call out of order (e.g. before gdfv_prepare) */

/* Face numbering of a structured block, src/geom/elements/nomenclature.d:12-19. */
#define GDFV_WEST 0
#define GDFV_EAST 1
#define GDFV_SOUTH 2
#define GDFV_NORTH 3
#define GDFV_BOTTOM 4
#define GDFV_TOP 5

/* New context on the current CUDA device; returns a handle >= 0 or < 0.
 * Replaces the global configuration object GlobalConfig (e4/globalconfig.d:927). */
int gdfv_context_new(void);
int gdfv_context_free(int ctx);

/* Solver options by the reference's own JSON/Lua key names and values
 * (e4/globalconfig.d:1858-2004 readers, :186-206 and :320-345 name->enum maps,
 * '-' accepted for '_').  Strings: flux_calculator (ausmdv | hllc | hlle),
 * gasdynamic_update_scheme (predictor_corrector | pc), thermo_interpolator (rhou),
 * flux_precision (fp64 | fp32), van_albada_variant (e4 | lmr: the limiter epsilon
 * scaled per face by the larger state beside it and the face's length factor, as
 * lmr/onedinterp.d:147-151 does; no e4 counterpart).  Integers: interpolation_order (2), dimensions (2|3),
 * MHD, divergence_cleaning, apply_limiter, extrema_clipping, apply_entropy_fix,
 * interpolate_in_local_frame (1), stringent_cfl, cfl_count, max_attempts_for_step,
 * max_invalid_cells, fixed_time_step, n_ghost_cell_layers (2), glm_reference_indexing,
 * tile_kchunk.  Doubles: cfl_value, dt_init, dt_max, epsilon_van_albada, R, gamma,
 * divB_damping_length, flowstate_limits_max_velocity, flowstate_limits_max_temp,
 * flowstate_limits_min_temp.  Unknown key or value: GDFV_ERR_ARG.
 * Scheduling integers with no reference counterpart (results do not depend on them):
 * tile_kchunk (planes per tile, 0: the block's nkc up to 32), persistent (1: each
 * stage is one resident grid taking the tiles of all blocks from a queue; default 0:
 * one CTA per tile), tile_width (float-flux Euler defaults: 32, the default, tiles 32
 * cells wide, one row per warp; 16: tiles 16 wide with two rows per warp, which leave
 * fewer lanes idle on blocks whose width is not a multiple of 32),
 * autotune (1: the first gdfv_run times the tile k-chunks, both launch forms and both
 * tile widths, and keeps the fastest).  gdfv_config_get_double also reads
 * tile_kchunk, persistent, tile_width, autotune and autotune_stage_ms (stage 1 + stage 2 time of the tuned choice), and after
 * gdfv_prepare tile_rows and tile_rows_corrector (rows per column tile of the stages
 * and of the corrector, which may take taller or shorter tiles of its own). */
int gdfv_config_set_str(int ctx, const char* key, const char* value);
int gdfv_config_set_int(int ctx, const char* key, long long value);
int gdfv_config_set_double(int ctx, const char* key, double value);
int gdfv_config_get_double(int ctx, const char* key, double* value);

/* A uniform Cartesian structured block of nic x njc x nkc cells with origin
 * (x0,y0,z0); returns the block id (>= 0).  Replaces SFluidBlock construction
 * (e4/sfluidblock.d:440-700) for axis-aligned grids. */
int gdfv_block_new(int ctx, int nic, int njc, int nkc, double dx, double dy, double dz,
                   double x0, double y0, double z0);

/* A rectilinear structured block of nic x njc x nkc cells from its vertex coordinates
 * along each axis (xv: nic+1, yv: njc+1, zv: nkc+1 values, increasing; 2D: zv two values):
 * cell (i, j, k) spans [xv[i], xv[i+1]] x [yv[j], yv[j+1]] x [zv[k], zv[k+1]]; returns
 * the block id.  Replaces SFluidBlock construction from a StructuredGrid
 * (e4/sfluidblock.d:440-700, geometry of src/geom/elements/properties.d:97-140) for
 * axis-aligned grids with stretched spacing: face areas and volumes are products of the
 * cell's lengths, the l2r2 weights come from the lengths of the cells in each stencil
 * (e4/onedinterp.d:338-355; ghost cells take the lengths of interior cell n, or of the
 * partner's cell across an exchange, e4/sfluidblock.d:884-1090), and the CFL signal
 * takes each cell's own lengths (e4/fvcell.d:975-1059).  Not with MHD or
 * van_albada_variant=lmr; the adjoint takes them (per-cell weights, areas and volumes). */
int gdfv_block_new_graded(int ctx, int nic, int njc, int nkc, const double* xv, const double* yv,
                          const double* zv);

/* Boundary condition of one face, by the reference's BC type names:
 *   "wall_with_slip"             WallBC_WithSlip (e4/bc.lua:733-757)
 *   "outflow_simple_extrapolate" OutFlowBC_SimpleExtrapolate, x_order 0 or 1 (:1511-1530)
 *   "inflow_supersonic"          InFlowBC_Supersonic; inflow = {p, T, vel.x, vel.y, vel.z,
 *                                B.x, B.y, B.z, psi} as FlowState:new{p=,T=,...} (:1251-1280)
 *   "exchange_over_full_face"    ExchangeBC_FullFace (:1603-1625) with orientation 0 onto
 *                                face other_face of block other_blk (any face: the ghost
 *                                cells copy the partner's cells inside that face); for
 *                                another orientation or a rotation see
 *                                gdfv_block_set_exchange
 *   "outflow_simple_flux"        OutFlowBC_SimpleFlux (:1532-1556): ghosts copy the boundary
 *                                cell, the boundary face's flux is the interior cell's
 *                                (boundary_flux_effect.d:504-645); not with MHD
 *   "outflow_fixed_p"            OutFlowBC_FixedP (:1558-1578), inflow = {p_outside}
 *   "outflow_fixed_p_and_t"      OutFlowBC_FixedPT (:1580-1600), inflow = {p_outside, T_outside}
 * Ghost cells are never stored: the kernels synthesise them (ghost_cell_effect/*.d). */
int gdfv_block_set_bc(int ctx, int blk, int face, const char* bc_type, int x_order,
                      int other_blk, int other_face, const double* inflow);

/* ExchangeBC_FullFace{otherBlock, otherFace, orientation, reorient_vector_quantities,
 * Rmatrix} (e4/bc.lua:1603-1625) on face `face` of block `blk`.  The ghost cell at depth
 * n beyond the face copies the partner's cell n layers inside face other_face, at the
 * tangential position that GhostCellFullFaceCopy.set_up_cell_mapping_phase0 gives for
 * the face pair and orientation 0..3 (e4/bc/ghost_cell_effect/full_face_copy.d:680-1409;
 * 2D blocks ignore the orientation, as there); gdfv_exchange_source evaluates that map.
 * Rmatrix: NULL, or 9 doubles (row major) applied to the ghost's velocity and magnetic
 * field (flowstate.d:393-400 reorient_vector_quantities, full_face_copy.d:2403-2405).
 * The faces' cell counts must match under the map and the partner must be at least 2
 * cells deep; checked at gdfv_prepare.  The adjoint follows both the map and the rotation. */
int gdfv_block_set_exchange(int ctx, int blk, int face, int other_blk, int other_face, int orientation,
                            const double* Rmatrix);

/* The partner cell that feeds a ghost cell of an exchange face, by the map above, without
 * a context: dims 2 or 3, faces 0..5 (0..3 in 2D), n_other = the partner's cell counts,
 * ijk = the ghost cell's indices in its own block (one index outside [0, n), at depth 0
 * or 1 beyond `face`); writes the partner's cell indices to src.  Returns GDFV_OK, or
 * GDFV_ERR_ARG for a bad face, orientation or ghost position. */
int gdfv_exchange_source(int dims, int face, int other_face, int orientation, const int* n_this,
                         const int* n_other, const int* ijk, int* src);

/* Validate the configuration and allocate device memory.  After this call
 * blocks and options are frozen. */
int gdfv_prepare(int ctx);

/* Initial state from host rhoT arrays (e4/fvcell.d:511-583 encode_conserved after
 * update_thermo_from_rhoT, ideal_gas.d:107-115). */
int gdfv_block_set_flow_rhoT(int ctx, int blk, const double* rhoT_host);
/* Conserved state of one block, host arrays. */
int gdfv_block_set_conserved(int ctx, int blk, const double* U_host);
int gdfv_block_get_conserved(int ctx, int blk, double* U_host);
/* Decoded flow state of one block (e4/fvcell.d:586-822 decode_conserved), host array. */
int gdfv_block_get_flow(int ctx, int blk, double* flow_host);
/* Number of cells in one block, and in all blocks together. */
long long gdfv_block_ncells(int ctx, int blk);
long long gdfv_total_cells(int ctx);

/* Time-march: take steps until max_steps more steps are done or time >= max_time
 * (max_time <= 0: no time limit).  Replaces the loop of integrate_in_time
 * (e4/simcore.d:1055-1366) around gasdynamic_explicit_increment_with_fixed_grid
 * (e4/simcore_gasdynamic_step.d:904-1587) with determine_time_step_size (:60-160)
 * and update_ch_for_divergence_cleaning (e4/simcore.d:1625-1648).  The dt rule, the
 * retry with dt*0.2 and the bad-cell abort run on the device.
 * Returns 0, GDFV_ERR_BAD_CELLS or GDFV_ERR_STEP_FAILED. */
int gdfv_run(int ctx, int max_steps, double max_time, int* steps_taken);
/* Where the last failed step failed: block id, (i, j, k) within the block and the
 * cell-centre position (x, y, z) of the failing cell with the lowest index among the
 * cells that failed to decode or failed check_data in the step's last attempt.  The
 * reference names that cell in its exceptions and reports: decode_conserved's "Bad
 * cell" (e4/fvcell.d:610-640: blk-id, cell-id, x, y, z) and count_invalid_cells
 * (e4/fluidblock.d:607-675); the error message of the failed call (gdfv_run,
 * gdfv_step_dt, gdfv_steps_dt, gdfv_step_noalloc) carries the same, with the cell id
 * i + nic (j + njc k).  Any pointer may be NULL.  GDFV_ERR_STATE when no failed step
 * has reported a cell. */
int gdfv_last_bad_cell(int ctx, int* blk, int* ijk, double* pos);

/* Replace the state of supersonic-inflow face `index` (faces numbered in the order
 * gdfv_block_set_bc defined them) after gdfv_prepare: state = {p, T, vel.x, vel.y,
 * vel.z, B.x, B.y, B.z, psi} as for "inflow_supersonic".  The ghost state is the
 * FlowState that InFlowBC_Supersonic carries into FlowStateCopy
 * (e4/bc/ghost_cell_effect/flow_state_copy.d:92-107), built with FlowState:new{p=,T=};
 * the reference fixes it at preparation and has no run-time counterpart.  The next
 * step uses it (captured steps read it from device memory). */
int gdfv_set_inflow(int ctx, int index, const double* state);

/* out5 = {time, dt_global, c_h, cfl_max, dt_allow}; step = steps taken so far. */
int gdfv_get_time(int ctx, double* out5, int* step);
/* Set the simulation time, step counter and dt_global (e.g. after a restart). */
int gdfv_set_time(int ctx, double time, int step, double dt_global);

/* Residual R(U) = dU/dt for every block, device arrays over all blocks ([nq][total]).
 * One call = FluidBlock.applyPreReconAction + convective_flux_phase0
 * (e4/sfluidblock.d:2188-2245) + FVCell.time_derivatives (e4/fvcell.d:824-856)
 * on the state U.  Uses the context's current c_h. */
int gdfv_residual(int ctx, const double* U_dev, double* R_dev);

/* Jacobian-vector product of the residual as evalJacobianVecProd does it with the real
 * Frechet derivative (e4/steadystate_core.d:1878-1970): Jv = (R(U + sigma v) - R0)/sigma,
 * device arrays [nq][total].  R0_dev may be NULL (R(U) is then evaluated) or R(U) from
 * the caller (a Newton-Krylov loop holds it).  sigma <= 0 takes the Knoll-McHugh
 * perturbation (:3040-3078) sum(eps|U| + eps)/(N max(||v||, sqrt(eps))), eps = 1e-7,
 * returned in sigma_used (may be NULL). */
int gdfv_residual_jvp(int ctx, const double* U_dev, const double* v_dev, const double* R0_dev, double sigma,
                      double* Jv_dev, double* sigma_used);

/* Vector-Jacobian product of the residual: G = (dR/dU)^T W at the state U, device
 * arrays [nq][total] over all blocks (the adjoint of gdfv_residual, hand-written:
 * reverse of decode_conserved, interp_l2r2 and ausmdv or hllc, with the branches of
 * the primal values).  g_inflow_host (may be NULL) receives, per supersonic-inflow face
 * state in the order the faces were defined, the cotangent of its ghost state
 * (rho, vel.x, vel.y, vel.z, u, a), 6 doubles each (MHD: and B.x, B.y, B.z, psi, 10
 * each).  Euler (2D or 3D) with flux_calculator=ausmdv or hllc, van_albada_variant e4 or
 * lmr, uniform or graded blocks, every boundary condition of this library: exchanges of
 * any orientation with or without an Rmatrix (the cotangent goes back through its
 * transpose) and the outflow boundaries with their own ghost or flux rule included.
 * MHD with hlle and GLM, the context's current c_h held fixed, every boundary condition
 * the MHD forward takes except outflow_fixed_p and outflow_fixed_p_and_t
 * (GDFV_ERR_ARG).  It is the transpose of the Jacobian-vector products of
 * e4/steadystate_core.d:1870-2060 (evalJacobianVecProd), which it is checked against. */
int gdfv_residual_vjp(int ctx, const double* U_dev, const double* W_dev, double* G_dev, double* g_inflow_host);

/* One predictor-corrector step of a given dt from U_in_dev to U_out_dev (device arrays
 * [nq][total], distinct), without the dt rule: the recomputation step of a
 * checkpointed adjoint, bit-identical to the step gdfv_run took with that dt (MHD with
 * divergence cleaning: c_h from the signal of U_in_dev, as gdfv_run forms it).
 * U1_out_dev (may be NULL) receives the predictor state U1 = U0 + dt R(U0). */
int gdfv_step_dt(int ctx, const double* U_in_dev, double* U_out_dev, double dt, double* U1_out_dev);

/* n steps of gdfv_step_dt in a chain: step m takes dts[m] from the previous output
 * (U_in_dev for m = 0) to U_out_dev[m] (U_out_dev[n-1] may be NULL: the last step
 * then forms only its predictor state); U1_out_dev (may be NULL, or hold NULL
 * entries) receives the predictor states.  The recomputation of one checkpoint
 * segment, with one host synchronisation at the end; a failed step is reported
 * then (the steps after it do not write).  No reference counterpart: the
 * reference has no adjoint of the time-accurate solver. */
int gdfv_steps_dt(int ctx, const double* U_in_dev, double* const* U_out_dev, double* const* U1_out_dev,
                  const double* dts, int n);

/* Adjoint of one predictor-corrector step of frozen dt at the states U0 (step start)
 * and U1 (its predictor state): lam <- lam + mu + (dR/dU(U0))^T (dt/2 lam + dt mu)
 * with mu = (dR/dU(U1))^T (dt/2 lam), in place on the device array lam [nq][total].
 * The inflow ghost-state cotangents of both products are added into g_inflow_dev
 * (device, [n_inflow][6], MHD [n_inflow][10], caller-zeroed).  Enqueued on the
 * context's stream with no host synchronisation.  Same scope as gdfv_residual_vjp.
 * MHD with divergence cleaning: the step's c_h is formed from U0 as gdfv_run forms it
 * (the signal of the step's start state) and held fixed; the corrector's read of U1
 * with psi damped, and the damping of U2's psi, are reversed.  No reference
 * counterpart. */
int gdfv_step_adjoint(int ctx, const double* U0_dev, const double* U1_dev, double dt, double* lam_dev,
                      double* g_inflow_dev);

/* The whole backward of a checkpointed rollout of nsteps predictor-corrector steps:
 * lam (device, [nq][total]) holds dJ/dU_N on entry and dJ/dU_0 on return, the inflow
 * cotangents are added into g_inflow_dev.  ckpt_dev[s] is the state at step
 * s*checkpoint_every (checkpoint_every <= 64; n_ckpt = ceil(nsteps/checkpoint_every) of them), dts the dt of
 * every step, work_dev 4*checkpoint_every state-sized device arrays: two sets of
 * (checkpoint_every states after steps, checkpoint_every predictor states).  Each
 * segment is recomputed (as gdfv_steps_dt) on a second stream while the adjoint steps
 * of the segment after it (as gdfv_step_adjoint) run on the context's stream; returns
 * after both finish.  last_ready != 0: the first set already holds the last
 * segment's states and predictor states (kept by the forward pass, see
 * gdfv_last_predictor_state), which are then not recomputed.  Same scope as
 * gdfv_step_adjoint; no reference counterpart. */
int gdfv_rollout_adjoint(int ctx, const double* const* ckpt_dev, int n_ckpt, const double* dts, int nsteps,
                         int checkpoint_every, double* const* work_dev, int last_ready, double* lam_dev,
                         double* g_inflow_dev);

/* nsteps steps as gdfv_run takes them (the dt rule on the device), each recorded on the
 * device as it completes, with no host round trip between steps: states_dev[n] (NULL:
 * not kept) receives the state after step n, preds_dev[n] (NULL: not kept) its
 * predictor state U1 = U0 + dt*dU0 (as gdfv_last_predictor_state forms it), and dts[n]
 * (host) its dt; device arrays [nq][total].  What a differentiable rollout keeps of its
 * trajectory.  A step that needed a retry leaves the record incomplete: GDFV_ERR_STATE,
 * with the state moved on.  No reference counterpart. */
int gdfv_run_record(int ctx, int nsteps, double* const* states_dev, double* const* preds_dev, double* dts);

/* Predictor state U1 = U0 + dt*dU0 of the step gdfv_run took last, from the state U0
 * before it (device arrays): what a forward pass keeps to differentiate its last
 * steps without recomputing them.  Valid directly after the step.  No reference
 * counterpart. */
int gdfv_last_predictor_state(int ctx, const double* U0_dev, double* U1_out_dev);

/* Residual norms of the step gdfv_run took last, as Eilmer reports them with
 * report_residuals (e4/simcore.d:1193-1195, :1212): Linf[q] = max over all cells of
 * |dU/dt[q]| of the step's predictor stage, q < nq
 * (FluidBlock.compute_Linf_residuals, e4/fluidblock.d:861-876, max over blocks
 * e4/simcore.d:1683-1695); L2 = sqrt of the sum over all cells of the squares of
 * mass, x and y momentum, z momentum (3D), total energy and, with MHD, xB and yB
 * (FluidBlock.compute_L2_residual, e4/fluidblock.d:879-909, summed over blocks
 * e4/simcore.d:1697-1706).  Linf may be NULL.  Reduced on the device (warp shuffles,
 * then the per-CTA partials in a fixed order); waits for the context's stream.
 * gdfv_step_dt, gdfv_steps_dt and gdfv_time_stages overwrite the predictor
 * derivative these norms are taken of. */
int gdfv_residual_norms(int ctx, double* Linf, double* L2);

/* Device pointer of the current conserved state ([nq][total], borrowed, valid
 * until the next gdfv_run), and of the context's CUDA stream. */
int gdfv_state_device_ptr(int ctx, double** U_dev);
int gdfv_set_stream(int ctx, void* cuda_stream);

/* Kernel timing: run `reps` repetitions of each stage kernel on the current state
 * without advancing it; ms[0] = stage 1, ms[1] = stage 2 average milliseconds per launch. */
int gdfv_time_stages(int ctx, int reps, double* ms);

/* One predictor-corrector step of size dt from U_in_dev to U_out_dev (device arrays
 * [nq][total], distinct), allocating no device memory.  This entry point has no
 * counterpart in the reference.  It is for callers that cannot call cudaMalloc: an
 * application whose device memory belongs to its own pool allocator, or a real-time
 * loop that cannot accept cudaMalloc's latency and implicit synchronisation.  The
 * step's scratch (predictor derivative, step-control record, signal maxima) lives in
 * one fixed device array that the library reserves on every GPU it is loaded on and
 * keeps until exit: nq * total cells must not exceed GDFV_NOALLOC_MAX_VALUES and the
 * blocks must not exceed GDFV_NOALLOC_MAX_BLOCKS, else GDFV_ERR_ARG.  All calls share
 * that array, so calls whose kernels overlap on the GPU race; calls made one after
 * another on the context's stream are safe.  The first call on a device looks up the
 * array's address; make it before any stream capture starts on that device (after a
 * device reset the address is looked up again).  MHD runs with divergence cleaning
 * take c_h by the rule of a gdfv_run step from the signal frequency of U_in (reduced
 * into the same scratch).  n_bad_cells (may be NULL) receives the decode failures plus
 * invalid cells; a decode failure returns GDFV_ERR_STEP_FAILED (no retry is
 * attempted); gdfv_last_bad_cell then locates the failing cell. */
#define GDFV_NOALLOC_MAX_VALUES 4194304LL
#define GDFV_NOALLOC_MAX_BLOCKS 1024
int gdfv_step_noalloc(int ctx, const double* U_in_dev, double* U_out_dev, double dt, int* n_bad_cells);

/* Copy of the last error message of a context (NUL-terminated, truncated to n). */
int gdfv_last_error(int ctx, char* buf, int n);

#ifdef __cplusplus
}
#endif
#endif /* GDFV_H */
