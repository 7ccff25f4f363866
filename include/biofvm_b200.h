/*
 * biofvm_b200.h -- C ABI of the B200-native BioFVM-B diffusion-decay path.
 *
 * One `bfb_env` is one device-resident microenvironment: a uniform Cartesian
 * voxel grid (nx, ny, nz) of edge dx holding S substrates, stored on the GPU in
 * the reference's layout  rho[((i*ny + j)*nz + k)*S + d]  (voxel-major,
 * substrate-inner; BioFVM_mesh.cpp:659-665), in FP64 or FP32.
 *
 * Every entry point returns an int status (BFB_OK = 0, negative on error) and
 * never aborts; bfb_last_error() gives the calling thread's last message.
 * Handles are not thread-safe; all device work of a handle is issued on its
 * stream (bfb_set_stream), so calls may be captured in a CUDA graph by the
 * caller. Host pointers are plain host memory (pinned memory makes the copies
 * asynchronous-capable but is not required). No torch types cross this line.
 *
 * Reference interfaces replaced (reference paths, file:line):
 *   - the swappable solver pointer  void (*diffusion_decay_solver)(Microenvironment&,
 *     double dt, int, int, int*, int*, MPI_Comm)   BioFVM_microenvironment.h:164,
 *     its callers simulate_diffusion_decay         BioFVM_microenvironment.cpp:1018-1029,
 *     and the solvers behind it                    BioFVM_parallel.cpp:693-1395 / 1411-2326
 *   - apply_dirichlet_conditions + Dirichlet setters
 *                                                  BioFVM_microenvironment.cpp:226-484
 *   - simulate_bulk_sources_and_sinks              BioFVM_microenvironment.cpp:1110-1153
 *   - simulate_cell_sources_and_sinks / Basic_Agent::simulate_secretion_and_uptake
 *                                                  BioFVM_microenvironment.cpp:1155-1169,
 *                                                  BioFVM_basic_agent.cpp:279-300
 */
#ifndef BIOFVM_B200_H
#define BIOFVM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BFB_API __attribute__((visibility("default")))
#else
#define BFB_API
#endif

typedef struct bfb_env_s *bfb_env;

/* status codes */
#define BFB_OK 0
#define BFB_ERR_INVALID_ARG (-1)
#define BFB_ERR_SIZE (-2)
#define BFB_ERR_OOM (-3)
#define BFB_ERR_CUDA (-4)
#define BFB_ERR_STATE (-5)
#define BFB_ERR_WATCHDOG (-6)
#define BFB_ERR_UNSUPPORTED (-7)

/* field precision */
#define BFB_FP64 0
#define BFB_FP32 1

/* options (bfb_set_option) */
#define BFB_OPT_FREEZE_FACTORS 1 /* 1 (default): Thomas factors are computed on the first step
                                    and kept, as BioFVM_parallel.cpp:714,913 does; 0: recomputed
                                    whenever dt differs from the cached one */
#define BFB_OPT_USE_GRAPHS 2     /* 1 (default): bfb_simulate replays a captured CUDA graph */
#define BFB_OPT_USE_TMA 3        /* 1 (default): sweeps move data with the TMA engine where the
                                    grid's row pitch allows; 0: cp.async kernels everywhere */

/* bfb_simulate flags: per step, in the order of examples/3D_tumor_example_X.cpp:346-348 */
#define BFB_STEP_BULK 1
#define BFB_STEP_DIFFUSION 2
#define BFB_STEP_CELLS 4

/* Thread-local text of the last error (never NULL). */
BFB_API const char *bfb_last_error(void);
BFB_API int bfb_version(void);

/* Create a grid of nx*ny*nz voxels of edge dx with S substrates whose domain
 * starts at the origin. Replaces Microenvironment() + resize_space_uniform()
 * (BioFVM_microenvironment.cpp:140-216, BioFVM_parallel.cpp:18-59) at one rank.
 * All D and lambda start at 0; no Dirichlet face is active (see
 * bfb_set_dirichlet for the reference's defaults). */
BFB_API int bfb_create(bfb_env *out, int nx, int ny, int nz, int n_substrates, double dx,
                       int precision, int device);

/* Same, from a domain box, with the reference's node count
 * n = (int)ceil(1e-16 + (hi - lo)/dx) per axis (BioFVM_parallel.cpp:100-102).
 * The box is also the one agent positions are binned against. */
BFB_API int bfb_create_domain(bfb_env *out, double x0, double x1, double y0, double y1,
                              double z0, double z1, double dx, int n_substrates, int precision,
                              int device);

BFB_API int bfb_destroy(bfb_env env);
BFB_API int bfb_get_shape(bfb_env env, int *nx, int *ny, int *nz, int *n_substrates);
/* Every env owns a non-blocking stream; bfb_set_stream(env, s) issues its
 * work on the caller's stream s instead (NULL: back to the env's own). */
BFB_API int bfb_set_stream(bfb_env env, void *cuda_stream);
BFB_API int bfb_set_option(bfb_env env, int option, int value);
BFB_API int bfb_synchronize(bfb_env env);
/* No counterpart in the reference (which has no device waits). Every wait of
 * the TMA kernels on a copy is bounded; one that runs out sets the env's
 * sticky error flag, after which bfb_synchronize, bfb_get_field[_raw],
 * bfb_step_host (which then leaves the host field unchanged), bfb_checksum,
 * bfb_get_gradients and bfb_write_matlab return BFB_ERR_WATCHDOG for this env.
 * bfb_watchdog_selftest queues, on the env's stream, one such wait (`polls`
 * polls, 1..2^20) on a barrier that nothing completes, so the error path can
 * be tested without stalling any copy; the flag stays set for the env's life. */
BFB_API int bfb_watchdog_selftest(bfb_env env, int polls);

/* Per-substrate diffusion coefficients and decay rates (the public vectors
 * diffusion_coefficients / decay_rates, BioFVM_microenvironment.h:151-152).
 * Invalidates the cached Thomas factors. */
BFB_API int bfb_set_coefficients(bfb_env env, const double *D, const double *lambda);

/* Field transfer, V*S values in the reference layout. The double variants
 * convert to/from the env's precision on the device; the _raw variants copy
 * the env's own element type (double for FP64, float for FP32). */
BFB_API int bfb_set_field(bfb_env env, const double *host);
BFB_API int bfb_get_field(bfb_env env, double *host);
BFB_API int bfb_set_field_raw(bfb_env env, const void *host);
BFB_API int bfb_get_field_raw(bfb_env env, void *host);
/* Device-to-device transfer of the field, converting from/to src/dst
 * precision (BFB_FP64 / BFB_FP32); src/dst hold V*S elements on the env's
 * device. The copy is ordered on the env's stream only: work that produces
 * src on another stream must be complete (or that stream given to
 * bfb_set_stream) before the call. Both calls return after the copy. */
BFB_API int bfb_set_field_device(bfb_env env, const void *src, int src_precision);
BFB_API int bfb_get_field_device(bfb_env env, void *dst, int dst_precision);
/* Error of one env's field against another's of the same shape (any
 * precisions): out4 = {max|a-b|, max|b|, sum (a-b)^2, sum b^2}, accumulated
 * in FP64 on the device. Relative L-inf = out4[0]/out4[1], relative
 * L2 = sqrt(out4[2]/out4[3]). */
BFB_API int bfb_compare_fields(bfb_env test, bfb_env ref, double *out4);
/* Device pointer of the field (env precision); valid until bfb_destroy.
 * Voxel (i, j, k), substrate d is element (i*ny + j)*Lp + k*S + d, Lp from
 * bfb_field_pitch: nz*S (the packed reference layout) unless nz*S elements
 * are not a whole number of 16-byte vectors, when each (i, j) row is padded
 * to the next 16 bytes (the tensor-tile copies need 16-byte row pitches).
 * Padding entries are not part of the field; the transfer calls above take
 * and return the packed layout. */
BFB_API int bfb_field_device_ptr(bfb_env env, void **dptr);
BFB_API int bfb_field_pitch(bfb_env env, int *row_elems);

/* Dirichlet conditions on the outer faces.
 *   values     V*S per-voxel values like the reference's dirichlet_value_vectors
 *              (only outer-face voxels are read), or NULL to keep the current ones
 *   activation S flags, dirichlet_activation_vector (BioFVM_microenvironment.cpp:328-332)
 *   face_mask  6*S flags [face][d] (faces x-lo, x-hi, y-lo, y-hi, z-lo, z-hi), or
 *              NULL for the reference's rule: all six faces follow activation[d]
 *              (BioFVM_microenvironment.cpp:381-484). A non-NULL mask is ANDed
 *              with activation and extends the reference (e.g. x-faces only).
 * A new env has every face inactive and all values 0; the reference's own
 * constructor defaults (activation true, value 100.0 after resize,
 * BioFVM_parallel.cpp:56) are applied by the C++ facade. */
BFB_API int bfb_set_dirichlet(bfb_env env, const double *values, const uint8_t *activation,
                              const uint8_t *face_mask);
/* set_substrate_dirichlet_value(d, v) for every d at once
 * (BioFVM_microenvironment.cpp:334-359): one value per substrate on all faces. */
BFB_API int bfb_set_dirichlet_uniform(bfb_env env, const double *value_per_substrate,
                                      const uint8_t *activation, const uint8_t *face_mask);
/* apply_dirichlet_conditions(rank, size) at one rank. */
BFB_API int bfb_apply_dirichlet(bfb_env env);

/* n_steps LOD diffusion-decay steps (Dir, X, Dir, Y, Dir, Z, Dir each),
 * the work of diffusion_decay_solver__constant_coefficients_LOD_3D. */
BFB_API int bfb_diffusion_step(bfb_env env, double dt, int n_steps);

/* Bulk sources and sinks: S (supply rate), T (target density), U (uptake
 * rate), V*S each, as the three bulk callbacks would write them
 * (BioFVM_microenvironment.h:165-167). Pass all NULL to disable. */
BFB_API int bfb_set_bulk(bfb_env env, const double *supply_rate, const double *target,
                         const double *uptake);
BFB_API int bfb_bulk_step(bfb_env env, double dt);

/* Agents (Basic_Agent): n agents in list order, pos n*3, volume n, rates n*S,
 * active n flags (NULL = all active). Binning, the cached constants of
 * set_internal_uptake_constants(dt) and the voxel sort run on the device. */
BFB_API int bfb_set_agents(bfb_env env, int n, const double *pos, const double *volume,
                           const double *secretion, const double *uptake,
                           const double *saturation, const uint8_t *active, double dt);
/* Agents from the state a Basic_Agent caches: current_voxel_index (n), and
 * cell_source_sink_solver_temp1/temp2 (n*S) of set_internal_uptake_constants
 * (BioFVM_basic_agent.cpp:155-176), in list order; active n flags or NULL.
 * Used by callers that keep the reference's agent objects and their lazily
 * refreshed constants (the C++ facade does). Voxels of active agents must lie
 * in [0, V). */
BFB_API int bfb_set_agent_constants(bfb_env env, int n, const int *voxel, const double *temp1,
                                    const double *temp2, const uint8_t *active);
/* current_voxel_index of each agent (list order). */
BFB_API int bfb_agent_voxels(bfb_env env, int *out);
BFB_API int bfb_cells_step(bfb_env env, double dt);

/* n_steps composite steps, each [bulk] -> [diffusion] -> [cells] by flags. */
BFB_API int bfb_simulate(bfb_env env, double dt, int n_steps, int flags);

/* Host-buffer step for reference-facing callers: copies host (V*S doubles)
 * to the device, runs n_steps diffusion steps, copies the result back. */
BFB_API int bfb_step_host(bfb_env env, double *host_field, double dt, int n_steps);

/* No counterpart in the reference. Page-locks (cudaHostRegister) `bytes` of
 * caller-owned host memory at `host`, such as a Microenvironment's field
 * vector, so that bfb_step_host / bfb_set_field / bfb_get_field copy it at
 * pinned-memory speed instead of through the driver's staging buffers.
 * bfb_host_unregister undoes it; call it before the memory is freed or
 * reallocated (for a std::vector: before it grows or is destroyed). */
BFB_API int bfb_host_register(void *host, size_t bytes);
BFB_API int bfb_host_unregister(void *host);

/* Device time per phase, the counterpart of the reference's -DTIMING per-sweep
 * CSV (BioFVM_parallel.cpp:695-697, 1259-1392): runs n_steps steps like
 * bfb_simulate (without a graph) with CUDA events around every launch and
 * adds the milliseconds of each phase to ms_out[BFB_PROFILE_PHASES]:
 * 0 x-sweep (with the fused pre-x Dirichlet / bulk), 1 y-sweep, 2 z-sweep,
 * 3 standalone bulk, 4 cells. */
#define BFB_PROFILE_PHASES 5
BFB_API int bfb_profile_steps(bfb_env env, double dt, int n_steps, int flags, double *ms_out);

/* ---- Launch-shape tuning -------------------------------------------------
 * No counterpart in the reference. The launch shape of the x, y and z sweeps:
 * shape[3*axis + 0] = 1 for TMA tiles (where the grid allows them), 0 for
 * cp.async tiles, 2 (FP64 x and y sweeps, lines of 16 to 256 rows; else as 1)
 * for TMA tiles whose lines' forward results are held in tensor memory;
 * shape[3*axis + 1] = warps (tiles) per CTA, 1..4;
 * shape[3*axis + 2] = row groups per TMA tile (pipeline stages), 1..16
 * (the tensor-memory tiles keep their own: 4 warps, 16-row groups).
 * Every shape computes the same numbers (FP64 bit for bit); only the speed
 * differs. Defaults {1, 1, 2} per axis. bfb_autotune times each candidate
 * (TMA / cp.async x 1, 2, 4 warps x 2, 4, 8 row groups; not the
 * tensor-memory tiles, which measured slower on every grid tried) of each
 * sweep with
 * CUDA events over `trials` launches, out of place from the env's field into
 * a scratch field (the field is unchanged; the scratch is freed on return),
 * keeps the fastest and returns it in chosen[BFB_TUNING_FIELDS] and its
 * milliseconds per launch in best_ms[3] (either may be NULL). */
#define BFB_TUNING_FIELDS 9
BFB_API int bfb_set_tuning(bfb_env env, const int *shape);
BFB_API int bfb_get_tuning(bfb_env env, int *shape);
BFB_API int bfb_autotune(bfb_env env, double dt, int trials, int *chosen, double *best_ms);

/* Gradient vectors of every substrate at every voxel, replacing
 * Microenvironment::compute_all_gradient_vectors (BioFVM_microenvironment.cpp:
 * 1243-1402) and the per-voxel compute_gradient_vector (:1404-1535), which
 * agree on the uniform mesh: out[(n*S + q)*3 + c] is the central difference
 * along axis c over 2*dx inside the grid and the one-sided difference over dx
 * at its two ends; 0 on an axis of one voxel. bfb_compute_gradients writes
 * 3*V*S elements of the env's precision to device memory, on the env's
 * stream (returns without waiting); bfb_get_gradients returns host doubles.
 * FP64 is bit-exact with the reference. An out_dev on a 16-byte boundary
 * (any cudaMalloc pointer) lets rows of a whole number of 16-byte vectors run
 * the faster vectorised kernel; other pointers give the same values. */
BFB_API int bfb_compute_gradients(bfb_env env, void *out_dev);
BFB_API int bfb_get_gradients(bfb_env env, double *out_host);

/* MATLAB v4 snapshot of the field, the file Microenvironment::write_to_matlab
 * writes (BioFVM_microenvironment.cpp:1079-1107, BioFVM_matlab.cpp:535-584;
 * BioFVM_parallel.cpp:528-678 at one rank): a (4 + S) x V double matrix named
 * "multiscale_microenvironment", one column per voxel holding the voxel
 * centre, its volume and its S densities. Packed on the device, copied to
 * pinned host memory and written; returns when the file is closed. FP64 files
 * are byte-identical to the reference's. */
BFB_API int bfb_write_matlab(bfb_env env, const char *filename);

/* Per-substrate FP64 sum of the field over all voxels (mass checksum). */
BFB_API int bfb_checksum(bfb_env env, double *out);

/* ---- Batched ensembles ---------------------------------------------------
 * Many independent envs (uneven shapes and substrate counts; one device and
 * one precision) stepped together: bfb_batch_simulate runs one LOD step of
 * every env -- and, with BFB_STEP_CELLS, its agents -- replayed from a CUDA
 * graph, in one of three modes:
 *   BFB_BATCH_MODE_STAGED (default): one launch per stage (x, y, z sweeps,
 *     agents), each a flat grid over every env's tiles, one warp per tile;
 *   BFB_BATCH_MODE_PERSISTENT: ONE persistent kernel launch per step whose
 *     warps pull (env, stage, tile) work items from a device queue;
 *   BFB_BATCH_MODE_GRAPH: every env's own step kernels (as bfb_simulate
 *     launches them), one independent branch per env of the step's graph,
 *     so the hardware schedules the envs' CTAs side by side.
 * The batch references the envs; they must outlive it, and their own settings
 * (coefficients, Dirichlet, agents) are the ones used.
 * bfb_batch_simulate_loop runs the same steps as one bfb_simulate call per
 * env (the per-instance launch loop). Not in the reference, which runs one
 * Microenvironment per MPI job. */
typedef struct bfb_batch_s *bfb_batch;
#define BFB_BATCH_OPT_WARPS_PER_CTA 1   /* 1..4, default 1 */
#define BFB_BATCH_OPT_TILES_PER_ITEM 2  /* warp tiles per queue item (persistent mode), 1..64, default 2 */
#define BFB_BATCH_OPT_MODE 3            /* BFB_BATCH_MODE_STAGED (default), _PERSISTENT or _GRAPH */
#define BFB_BATCH_MODE_PERSISTENT 0
#define BFB_BATCH_MODE_STAGED 1
#define BFB_BATCH_MODE_GRAPH 2
BFB_API int bfb_batch_create(bfb_batch *out, int n_envs, const bfb_env *envs);
BFB_API int bfb_batch_destroy(bfb_batch batch);
BFB_API int bfb_batch_set_option(bfb_batch batch, int option, int value);
BFB_API int bfb_batch_get_option(bfb_batch batch, int option, int *value);
BFB_API int bfb_batch_simulate(bfb_batch batch, double dt, int n_steps, int flags);
BFB_API int bfb_batch_simulate_loop(bfb_batch batch, double dt, int n_steps, int flags);
/* A batch owns a non-blocking stream; bfb_batch_set_stream issues its steps
 * (and orders bfb_batch_simulate_loop's per-env work) on the caller's stream
 * instead (NULL: back to its own), e.g. to time them with events there. */
BFB_API int bfb_batch_set_stream(bfb_batch batch, void *cuda_stream);
BFB_API int bfb_batch_synchronize(bfb_batch batch);
/* Times bfb_batch_simulate in the staged mode with warps per CTA {1, 2, 4},
 * in the persistent mode with warps per CTA {1, 2, 4} x tiles per item
 * {1, 2, 4, 8} and in the graph mode (8 warm steps and 8*`trials` timed
 * steps each, CUDA events; bfb_batch_simulate replays 8 steps per graph
 * launch while at least 8 remain), keeps the fastest and returns it in
 * chosen[2] = {warps, tiles per item} (the mode: bfb_batch_get_option with
 * BFB_BATCH_OPT_MODE) and its milliseconds per step in *best_ms (either may
 * be NULL). The trial steps advance the envs' fields, so every field is
 * saved first and restored before returning. Not in the reference. */
BFB_API int bfb_batch_autotune(bfb_batch batch, double dt, int flags, int trials, int *chosen, double *best_ms);

/* ---- Reverse mode ---------------------------------------------------------
 * No counterpart in the reference. Runs n_steps steps of `flags`
 * (BFB_STEP_DIFFUSION, optionally | BFB_STEP_CELLS) from the env's current
 * field, keeping a checkpoint every checkpoint_every steps, and returns the
 * gradients of a scalar loss L(final field) given dL/d(final field):
 *   dL_dfinal     device, N elements of the env precision (required)
 *   dL_dinitial   device, N elements: dL/d(initial field)         (or NULL)
 *   final_field   device, N elements: the field after n_steps     (or NULL)
 *   dL_dD, dL_dlambda              host, [S] doubles              (or NULL;
 *                 with both NULL the per-line sums they need are skipped,
 *                 about half of the reverse pass's memory traffic)
 *   dL_dsecretion, dL_duptake, dL_dsaturation
 *                 host, [n_agents][S] doubles in bfb_set_agents' list order
 *                 (or NULL); inactive agents get 0. They need the rates of
 *                 bfb_set_agents (BFB_ERR_STATE after bfb_set_agent_constants).
 * The derivative is that of the step as computed: the LOD splitting, the
 * active Dirichlet faces (their values are constants) and the agents'
 * implicit update, with the factors held at this dt. dL/dD and dL/dlambda are
 * summed in a fixed order (run-to-run identical). The env's field holds the
 * final field afterwards. The reverse pass recomputes each segment from its
 * checkpoint and keeps that segment's stage fields: device memory is about
 * (n_steps/checkpoint_every + 3*checkpoint_every + 3) fields. BFB_STEP_BULK is
 * not supported (BFB_ERR_UNSUPPORTED), nor lines whose two shared-memory tiles
 * exceed 227 KB (n*32*2 elements on x and y). Synchronous: returns when the
 * host gradients are written. */
BFB_API int bfb_adjoint_run(bfb_env env, double dt, int n_steps, int flags, int checkpoint_every,
                            const void *dL_dfinal, void *dL_dinitial, void *final_field, double *dL_dD,
                            double *dL_dlambda, double *dL_dsecretion, double *dL_duptake, double *dL_dsaturation);

/* No counterpart in the reference. The per-substrate FP64 sums of
 * bfb_checksum for callers that must not allocate device memory -- for
 * example code that owns its device buffers in its own pool, or a host loop
 * with other streams in flight, which cudaMalloc/cudaFree would stall by
 * synchronizing the device. The field is given directly: field_dev is a device
 * array of n_voxels*n_substrates elements in the reference layout, of
 * `precision` (BFB_FP64 / BFB_FP32); out_dev receives n_substrates doubles in
 * device memory. Work is queued on `stream` (NULL: the legacy default stream)
 * and the call returns without waiting. Its scratch is a fixed array inside
 * the library, so at most BFB_NOALLOC_MAX_SUBSTRATES substrates (larger counts
 * return BFB_ERR_SIZE), and calls that overlap on the GPU share that array and
 * race: order them on one stream. The first call on each device looks the
 * array's device address up (cudaGetSymbolAddress) and keeps it for the rest
 * of the process; make that first call before capturing a stream. The kept
 * address does not survive a reset of the device's primary context
 * (cudaDeviceReset): do not call this entry point after one. The call
 * allocates nothing. */
#define BFB_NOALLOC_MAX_SUBSTRATES 64
BFB_API int bfb_checksum_noalloc(const void *field_dev, int precision, long long n_voxels, int n_substrates,
                                 double *out_dev, void *stream);

/* ---- x-slab decomposition of one grid over ranks (FP64) -------------------
 * Replaces the reference's MPI split of the x planes (BioFVM_parallel.cpp:
 * 108-144, local counts x_nodes/dims[1]) and its pipelined cross-rank x solve
 * (BioFVM_parallel.cpp:948-1255 with the sends and receives of :832-873). A
 * slab env holds planes [x0, x0 + nx_local) of a grid of nx_global planes,
 * one rank (GPU) each; it is an ordinary env (field, Dirichlet, bulk, agents
 * of its own voxels; its domain box starts at x0*dx) whose x lines continue
 * in the neighbouring slabs. Its Dirichlet x faces are active only where the
 * slab holds the grid's face (x0 == 0 for the low face, x0 + nx_local ==
 * nx_global for the high one). A step is, per rank:
 *   bfb_slab_x_forward over line ranges, each after receiving prev_in for
 *     that range from the previous rank and followed by sending prev_out to
 *     the next;
 *   bfb_slab_x_backward over the ranges, each after receiving next_in from
 *     the next rank and followed by sending next_out to the previous;
 *   bfb_slab_yz.
 * Lines are the slab's columns, `lines` (bfb_slab_info) = ny * bfb_field_pitch
 * of them; prev_* / next_* are device arrays of `lines` doubles indexed by
 * line, of which [line0, line1) are read or written. prev_in is ignored on
 * the first slab and next_in on the last; prev_out / next_out may be NULL.
 * The slabs together give the whole grid's step bit for bit. bfb_simulate,
 * bfb_profile_steps, bfb_autotune, bfb_adjoint_run and batches refuse slab
 * envs (BFB_ERR_UNSUPPORTED). Work is queued on the env's stream. */
BFB_API int bfb_create_slab(bfb_env *out, int nx_global, int x0, int nx_local, int ny, int nz, int n_substrates,
                            double dx, int device);
BFB_API int bfb_slab_info(bfb_env env, int *nx_global, int *x0, long long *lines);
BFB_API int bfb_slab_x_forward(bfb_env env, double dt, const double *prev_in, double *prev_out, long long line0,
                               long long line1);
BFB_API int bfb_slab_x_backward(bfb_env env, double dt, const double *next_in, double *next_out, long long line0,
                                long long line1);
BFB_API int bfb_slab_yz(bfb_env env, double dt);

#ifdef __cplusplus
}
#endif
#endif
