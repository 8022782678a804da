/* cavity_solver.h - C ABI of the B200 cavity solver (libcavity_solver.so).
 *
 * Drop-in for the reference's ctypes boundary: the 18 `solver_*` functions below carry the names,
 * arguments, return codes and record layouts of backend.cu:983-1195 (Config / Report / Diagnostics:
 * backend.cu:584-597, mirrored by python_api.py:11-28).  Every function returns 0 on success and 1 on
 * error, with the message in solver_last_error().  As in the reference, they act on one process-wide
 * solver that solver_create replaces, every call is synchronous, and host buffers are caller-owned
 * with sizes implied by the grid (u: (nx+1)*ny*nz, v: nx*(ny+1)*nz, w: nx*ny*(nz+1), phi: nx*ny*nz).
 *
 * The `cavity_*` functions after them are additions with no counterpart in the reference (the
 * reference's solver is a singleton with one precision): a precision switch for the singleton and a
 * handle API for several independent cavities in one process.
 */
#ifndef CAVITY_SOLVER_H
#define CAVITY_SOLVER_H

#ifdef __cplusplus
extern "C" {
#endif

/* Solver settings; 288 bytes, first double at offset 48 (backend.cu:584-589). */
typedef struct CavityConfig {
    int nx, ny, nz, lid_shaped, impulse_order, adaptive_dt, dt_lag, phi_extrapolate, fdm_max_passes,
        grid_stretch, n_probes;
    double length, u_lid, nu, lz, lid_ramp_t, reinit_r, impulse_order4_ramp, grid_dx_wall, grid_max_aspect;
    double dt_fixed, dt_max, cfl_target, diffusion_limit, fdm_rtol;
    double probe_x[8], probe_y[8];
} CavityConfig;

/* Clock after a step; 48 bytes (backend.cu:590-594). dt_reason: 0 fixed, 1 DT_MAX, 2 CFL, 3 viscous. */
typedef struct CavityReport {
    long long steps;
    double time, dt, cfl, phi_rel;
    int dt_reason, phi_passes;
} CavityReport;

/* Volume-averaged diagnostics; 64 bytes (backend.cu:595-597). */
typedef struct CavityDiagnostics {
    double kinetic_energy, enstrophy, umax, div_rms, cfl_rate, gauge_ratio, gauge_x, gauge_y;
} CavityDiagnostics;

/* ---- the reference's boundary (backend.cu:1000-1195) ---- */
int solver_create(const CavityConfig* config);                              /* backend.cu:1009 */
int solver_initialize(const double* v_noise, const double* w_noise);        /* backend.cu:1075 */
int solver_step(CavityReport* report);                                      /* backend.cu:1089 */
int solver_kick(const double* nu, const double* nv, const double* nw, double amp, int passes); /* backend.cu:1092 */
int solver_report(CavityReport* report);                                    /* backend.cu:1095 */
int solver_diagnostics(CavityDiagnostics* d);                               /* backend.cu:1096 */
int solver_grid(int axis, double* faces, double* centres);                  /* backend.cu:1131 */
int solver_get_field(int field, void* out);                                 /* backend.cu:1139 */
int solver_set_field(int field, const void* in);                            /* backend.cu:1147 */
int solver_set_clock(double t, long long steps, double last_dt);            /* backend.cu:1156 */
int solver_probes(float* out);                                              /* backend.cu:1159 */
int solver_add_statistics(double weight, double* centreline);               /* backend.cu:1168 */
int solver_get_statistics(double* sums);                                    /* backend.cu:1176 */
int solver_set_statistics(const double* sums);                              /* backend.cu:1177 */
int solver_midplane(float* out);                                            /* backend.cu:1178 */
int solver_q_volume(int colour_w, float* q, float* colour);                 /* backend.cu:1185 */
int solver_destroy(void);                                                   /* backend.cu:1000 */
const char* solver_last_error(void);                                        /* backend.cu:1195 */

/* ---- additions (no counterpart in the reference) ---- */
/* Precision of the solver the next solver_create builds: 0 = FP64 fields (default), 1 = mixed (FP32
 * fields, FP64 pressure).  Returns 1 for any other value. */
int cavity_set_precision(int precision);

/* The current field of the process-wide solver in double (velocity and impulse are float32 in
 * solver_get_field); same numbering and sizes as solver_get_field. */
int cavity_get_field_f64(int field, double* out);

/* Handle API: several independent cavities.  A handle is an opaque pointer; the functions mirror the
 * solver_* ones above with the handle as first argument. */
typedef struct CavitySolver CavitySolver;
int cavity_create(const CavityConfig* config, int precision, CavitySolver** out);
int cavity_destroy(CavitySolver* s);
int cavity_initialize(CavitySolver* s, const double* v_noise, const double* w_noise);
int cavity_step(CavitySolver* s, CavityReport* report);
/* Enqueue `count` steps without waiting for the GPU; cavity_sync then waits, checks every step's status
 * and fills the report of the last one.  Steps of different handles overlap on the device. */
int cavity_step_async(CavitySolver* s, int count);
int cavity_sync(CavitySolver* s, CavityReport* report);
int cavity_get_field(CavitySolver* s, int field, void* out);
int cavity_set_field(CavitySolver* s, int field, const void* in);
/* Handle forms of solver_report and solver_set_clock (backend.cu:1092-1094, 1156-1158). */
int cavity_report(CavitySolver* s, CavityReport* r);
int cavity_set_clock(CavitySolver* s, double t, long long steps, double last_dt);
int cavity_probes(CavitySolver* s, float* out);
/* Handle forms of solver_add_statistics and solver_get_statistics (backend.cu:1168-1180). */
int cavity_add_statistics(CavitySolver* s, double weight, double* centreline);
int cavity_get_statistics(CavitySolver* s, double* sums);
int cavity_diagnostics(CavitySolver* s, CavityDiagnostics* d);
/* Device bytes this cavity holds (state, work arrays, pressure tables), for admission control. */
long long cavity_device_bytes(const CavitySolver* s);
/* Bytes a cavity of this config would hold, without creating it. */
long long cavity_estimate_bytes(const CavityConfig* config, int precision);

/* Timing support for benchmarks: run `warmup` untimed steps, then `steps` steps, each bracketed by CUDA
 * events on the solver's stream, with the L2 cache flushed (a 256 MiB device write) before each timed
 * step when flush_l2 != 0.  ms_per_step[steps] receives each step's device time.  When kernel_ms is not NULL,
 * `steps` more steps follow through a step graph that also records events around the kernels; kernel_ms[steps]
 * receives the device time of each one's momentum-sweep launches (see also cavity_kernel_times). */
int cavity_time_steps(CavitySolver* s, int warmup, int steps, int flush_l2, float* ms_per_step, float* kernel_ms);
/* Autotuner (no counterpart in the reference): times `steps` whole steps from the current state under each
 * candidate, restoring the state after each, and keeps the fastest for this cavity, in two rounds: the momentum
 * sweep (the tile kernel, in FP32 also its packed two-cells-per-thread form, or the z-march with 1/2, 1, 2 or 4
 * times its device-filling z-chunk count; only the
 * kernel CAVITY_SWEEP names, when set), then the FP64 transforms (six launches of 64 x 64 or 32 x 32 tiles, one
 * cooperative launch of 32 x 32 tiles, or, where no axis exceeds 64 cells, three launches of two chained
 * transforms each).  The choice is cached per grid size, stretching and precision form
 * for the process, and in the file named by CAVITY_TUNE_FILE when that is set; cavities created later with the
 * same key start with it.  The transform choices and the chunk counts give bit-identical steps; the two sweep
 * kernels agree to rounding.  With CAVITY_AUTOTUNE=1 a cavity without a cached choice tunes itself (6 steps per
 * candidate) before its first step.  Outputs (each may be NULL): the chosen chunk count (0: the tile sweep),
 * tile (0: the size rule) and pass form (0 six launches, 1 one cooperative launch, 2 three paired launches, -1
 * the size rule), and the step time in milliseconds. */
int cavity_autotune(CavitySolver* s, int steps, int* march_chunks, int* dgemm_tile, int* fused_pass, float* ms_per_step);
/* After cavity_time_steps: ms[5] receives the mean device time per timed step (milliseconds, all three stages)
 * of the momentum sweeps, the projection starts, the residuals of their warm-start guesses, the finishes, and
 * the six transforms of each stage's first pressure pass.  No counterpart in the reference. */
int cavity_kernel_times(CavitySolver* s, double* ms);
/* The generalised eigenbasis of one axis's pressure operator, K S = W S diag(lambda) with S^T W S = I, for the grid
 * that `config` describes along `axis` (0 x, 1 y, 2 z): lambda[n] (the constant mode set to 0) and the row-major
 * n x n S, eigenvector j in column j.  on_gpu = 0: implicit-shift QL on the host (the solvers' set-up); 1:
 * bisection and inverse iteration on the GPU (the solvers' set-up with CAVITY_EIGEN=gpu).  The eigenvectors'
 * order and signs differ between the two.  The reference computes this basis by
 * Jacobi rotations on the host (backend.cu:723-767); no counterpart of this function. */
int cavity_eigenbasis(const CavityConfig* config, int axis, int on_gpu, double* lambda, double* S);
/* The handle of the process-wide solver behind the solver_* functions (NULL if none). */
CavitySolver* cavity_default(void);
/* Number of kernels one step launches (fixed part plus per pressure pass, for the cavity's transform launches) for
 * the counts it reports. */
int cavity_kernels_per_step(const CavitySolver* s, int phi_passes_per_stage);
/* Queued steps with per-step outputs (no counterpart in the reference, whose run script makes a blocking
 * round trip per step for solver_probes and solver_add_statistics): queue `count` steps, each followed on the
 * device by its probe values (into a library-owned ring of pinned host memory, at most 4096 steps between
 * syncs) and, if `statistics`, by the mid-span statistics weighted with that step's dt.  cavity_sync_outputs
 * waits, fills the report, copies the probe values of up to max_steps queued steps (2*n_probes floats each,
 * in order) and stores their number in *steps_out. */
int cavity_step_outputs_async(CavitySolver* s, int count, int statistics);
int cavity_sync_outputs(CavitySolver* s, CavityReport* r, float* probes, int max_steps, int* steps_out);
/* Checkpoints (no counterpart in the reference, whose restart through solver_set_field drops the potential
 * history and the dt lag, backend.cu:1153): the complete state that decides the following steps (fields,
 * potential, the four potential-increment buffers, the control block with the history times, dt lag, CFL rate
 * and clock, and the statistics sums) copied to or from a caller-owned buffer of cavity_checkpoint_bytes
 * bytes, on the device (fast snapshots: *_is_device = 1) or on the host (persistence).  Continuing from a
 * loaded checkpoint is bit-identical to never having stopped.  A checkpoint loads only into a solver of the
 * same grid size and precision form; both calls require no queued steps. */
long long cavity_checkpoint_bytes(const CavitySolver* s);
int cavity_checkpoint_save(CavitySolver* s, void* dst, int dst_is_device);
int cavity_checkpoint_load(CavitySolver* s, const void* src, int src_is_device);
/* Batches (no counterpart in the reference): cavities of one precision form stepped together by one CUDA graph
 * per step, each of whose kernel launches covers every cavity through a work list of (cavity, block) entries,
 * so the cavities may differ in grid size.  Every cavity keeps its own dt, pass count, clock and errors, and
 * stays usable through its own handle between steps.  The members must have no queued steps when the batch is
 * created; take a cavity out of the batch (or destroy the batch) before destroying the cavity.
 * cavity_batch_sync waits for the queued steps and fills `reports` (one per slot, in order; an empty slot's
 * report is zero with steps = -1); if a member's step failed it reports that member's last good state and
 * returns 1 with the error, naming the slot.  A batch whose members' states have diverged (a failed step)
 * refuses further steps.
 * cavity_batch_create_slots makes a batch of `capacity` slots, the first `count` holding `members`, the rest
 * empty (the members then need one grid size).  cavity_batch_set_member puts a cavity of the batch's grid
 * size, form and kernels into a slot, or empties it (s = NULL), without rebuilding the batch's graphs: it
 * rewrites the slot's argument records and live flag in the device buffers the graphs read, so a served stream
 * of requests joins and leaves a running batch.  It needs no queued steps, and the cavity may be at either
 * state parity.  Blocks of an empty slot return at once. */
typedef struct CavityBatch CavityBatch;
int cavity_batch_create(CavitySolver* const* members, int count, CavityBatch** out);
int cavity_batch_create_slots(CavitySolver* const* members, int count, int capacity, CavityBatch** out);
int cavity_batch_set_member(CavityBatch* b, int slot, CavitySolver* s);
int cavity_batch_size(const CavityBatch* b);
/* Advances the batch `steps` steps through an instrumented copy of its step graph (built from the current members)
 * and fills ms[4] with the mean device time per step, in milliseconds summed over the three stages, of: the
 * momentum sweeps; the projection starts with the residuals of their warm-start guesses; each stage's first
 * pressure pass (transforms and residual; further passes, inside the refinement loop, are not timed); and the
 * finishes.  The steps are ordinary steps (the same kernels in the same order); no steps may be queued.  No
 * counterpart in the reference. */
int cavity_batch_part_times(CavityBatch* b, int steps, double* ms);
int cavity_batch_step_async(CavityBatch* b, int count);
int cavity_batch_sync(CavityBatch* b, CavityReport* reports);
int cavity_batch_destroy(CavityBatch* b);
/* One pass of the fast-diagonalisation pressure solve on caller-provided device arrays (the operation of
 * backend.cu:801-814 without the rms scaling): phi += S_x S_y S_z (inv_lambda .* (S_z^T S_y^T S_x^T r)), each
 * S applied along its axis.  s[a] / st[a]: the row-major n_a x n_a eigenbasis of axis a (eigenvector j in
 * column j) and its transpose; inv_lambda, r, phi: nx*ny*nz doubles, [z][y][x] with x fastest.  All are
 * device pointers.  Runs on `stream` (a cudaStream_t, NULL for the default stream), allocates its two
 * nx*ny*nz intermediates on that stream, and returns when phi is updated. */
int cavity_fdm_pass(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                    const double* inv_lambda, const double* r, double* phi, void* stream);
/* The mixed form's FDM pass on the tcgen05 tensor cores, on caller-provided device arrays: the operation of
 * backend.cu:801-814 with its scaling of r to rms 1, S and 1/lambda rounded to float (backend.cu:766-786)
 * and fp32 transforms, each computed as three TF32 products (3xTF32).  Same arguments as cavity_fdm_pass
 * (st is checked but not read: S^T is formed from s).  nx must be a multiple of 4.  Allocates its
 * intermediates on `stream` and returns when phi is updated. */
int cavity_fdm_pass_tf32(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                         const double* inv_lambda, const double* r, double* phi, void* stream);
/* cavity_fdm_pass without any device allocation (no counterpart in the reference).  For callers that must
 * not allocate device memory themselves or through this library: a host whose device memory is all owned
 * by its own pool allocator, or a process running with the device nearly full, where a cudaMalloc would
 * fail or a cudaFree would stall every stream.  Same arguments and result as cavity_fdm_pass; the caller
 * still passes every input and output.  The two intermediates live in a file-scope device array of
 * 2 x 262144 doubles (4 MiB, with a control block) that every GPU loading the library holds until the
 * process exits, so nx*ny*nz is limited to 262144 cells (64^3), and each axis to 1 <= n <= 1024 as for
 * cavity_fdm_pass; other grids are rejected with an error.  The first call on each device looks up the
 * array's device address once (set-up).  Every call is synchronous: it copies a control block from the
 * host and waits for `stream`, so it must not be called on a stream that is being captured.  All calls on a
 * device share the array, which keeps the last call's contents: each call resets the control flags that
 * must start at zero, and calls that overlap on the GPU race. */
int cavity_fdm_pass_noalloc(int nx, int ny, int nz, const double* const s[3], const double* const st[3],
                            const double* inv_lambda, const double* r, double* phi, void* stream);
/* Pressure passes run by this cavity since it was created (all stages, steps and projections). */
long long cavity_pressure_passes(const CavitySolver* s);
const char* cavity_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
