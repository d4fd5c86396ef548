/*
 * mun_sem.h — C ABI of the B200 (sm_100a) SEM forward/adjoint solver.
 *
 * This is the boundary that MUN's Python ``sem_waveform`` package would bind with
 * ctypes.  Every entry point replaces a piece of the reference's CPU path:
 *
 *   sem_plan_create     <- SEMSimulation._initialize_components
 *                          (Bspline_Coupling/SEM/sem_waveform/core.py:151-325): mesh,
 *                          GLL operators, lumped mass, sponge, source, receivers.
 *   sem_run             <- SEMSimulation.run / _time_stepping_loop_torch
 *                          (core.py:334-435, 598-659) and
 *                          SEMSimulation.run_forward_and_adjoint (core.py:1067-1371):
 *                          forward loop, misfit, adjoint loop and the per-step
 *                          sensitivity accumulate_sensitivity_dJdc_torch (core.py:49-85)
 *                          for one or many solves in one launch sequence.
 *   sem_forward         <- SEMSimulation.run (single solve convenience).
 *   sem_forward_adjoint <- SEMSimulation.run_forward_and_adjoint up to the node-space
 *                          gradient dJ_dv (core.py:1278), single solve.
 *
 * All device pointers are plain CUDA device addresses; ``stream`` is a cudaStream_t
 * passed as void*.  Calls are stream-ordered and return a status code.  A plan is
 * read-only after creation and may be shared by threads; a batch must be used by one
 * thread at a time (each thread uses its own batch).
 */
#ifndef MUN_SEM_H
#define MUN_SEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; the Python layer maps them to ValueError / RuntimeError / MemoryError */
enum {
  SEM_OK = 0,
  SEM_ERR_ARG = 1,        /* bad argument (reference: ValueError)                    */
  SEM_ERR_CUDA = 2,       /* CUDA runtime error                                      */
  SEM_ERR_OOM = 3,        /* device allocation failed                                */
  SEM_ERR_NONFINITE = 4,  /* NaN/Inf detected in a wavefield (reported per solve)    */
  SEM_ERR_TIMEOUT = 5,    /* a bounded device wait gave up                           */
  SEM_ERR_UNSUPPORTED = 6 /* polynomial order outside 1..7                           */
};

/* sem_solve_t.flags */
enum {
  SEM_F_ADJOINT = 1,  /* run the adjoint sweep and accumulate the gradient          */
  SEM_F_EXACT = 2,    /* apply the sponge inside the adjoint (exact discrete adjoint) */
  SEM_F_MISFIT = 4,   /* accumulate sum of squared residuals against y_obs          */
  SEM_F_SHIFT = 8     /* record R u after the update (run_forward_and_adjoint);
                         without it R u is recorded before the update (run())       */
};

typedef struct sem_plan_s sem_plan_t;
typedef struct sem_batch_s sem_batch_t;

/* Everything about one (mesh, order, dt, nt, source, receivers) signature.  All
 * arrays are HOST pointers to float64 (converted to float32 on upload).  nxg =
 * nelx*npol+1, nzg = nelz*npol+1. */
typedef struct {
  int32_t nelx, nelz, npol, nt;
  int32_t npoints;          /* number of mesh nodes = nxg*nzg                         */
  double dt;
  const int64_t* node_grid; /* [npoints] gz*nxg+gx of each node in reference order    */
  const double* gll_D;      /* [(npol+1)^2] D[a*(npol+1)+b] = l_b'(xi_a)              */
  const double* gll_beta;   /* [npol+1] w_a * l_a  (GLL weight x Lagrange quirk factor)*/
  const double* tab_x;      /* [3*nxg] 1/mx, Rx, 1 - sponge decay factor along x     */
  const double* tab_z;      /* [3*nzg] dt^2/(J mz), Rz, 1 - sponge decay along z     */
  const double* src_term;   /* [nt] dt^2 * s(t_it) added at the source node           */
  int32_t src_gx, src_gz;   /* source node (structured index)                         */
  int32_t nrec;
  const int32_t* rec_base;  /* [nrec*2] (gx0,gz0) first node of the receiver element  */
  const double* rec_w;      /* [nrec*(npol+1)^2] Lagrange weights, index j*(npol+1)+i */
  /* Boundary mode.  0: the reference's sponge (1 - its decay is the third row of tab_x and
   * tab_z).  1: an extension without counterpart in the reference: first-order Stacey
   * absorbing edges on the sides and the bottom and a free surface (u = 0) on the top row;
   * tab_x / tab_z then carry no decay (third rows 0).  The forward becomes
   *   (1 + a) u+ = 2 u - (1 - a) u- + dt^2 M^-1 (f - K u),  a = c alpha on the absorbing
   * edges, and the adjoint is its exact discrete adjoint: the same recurrence run
   * backwards, with a boundary-impedance term in the gradient (from d a / d c): at each
   * adjoint step the node of slot i adds (gamma_i / c_i) lambda_i (u_i(t+1) - u_i(t-1))
   * to the sensitivity of c_i^2.
   * Slots: (gx = 0, gz) -> gz, (gx = nxg-1, gz) -> nzg + gz, (gx, gz = nzg-1) -> 2 nzg + gx;
   * bnd_n = 2 nzg + nxg.  Ignored in mode 0. */
  int32_t boundary_mode;
  int32_t bnd_n;
  const int32_t* bnd_ref;   /* [bnd_n] reference node index of the slot's node, or -1   */
  const double* bnd_alpha;  /* [bnd_n] dt beta / (2 M): a = c alpha                     */
  const double* bnd_gamma;  /* [bnd_n] beta / (4 dt): impedance-term factor g = gamma/c */
} sem_plan_desc_t;

/* One solve inside sem_run.  Device pointers unless stated. */
typedef struct {
  const sem_plan_t* plan;
  const double* velocity;   /* [npoints] nodal velocity, reference node order         */
  int32_t flags;            /* SEM_F_*                                                */
  int32_t ckpt_k;           /* checkpoint interval for the adjoint replay (>=2); 0 =
                               automatic (see sem_launch_cfg_t.memory_budget)          */
  const double* y_obs;      /* [n_obs*nrec] observations on the misfit grid or NULL   */
  int32_t it0, it1, decim;  /* misfit window [it0,it1) and decimation (0,nt,1 = all)  */
  double inv_sigma2;        /* 1/(sigma^2 + 1e-24)                                    */
  float* rec_out;           /* [nt*nrec] receiver traces                              */
  double* loglik_out;       /* [1] -0.5*inv_sigma2*sum r^2 (SEM_F_MISFIT) or NULL     */
  double* grad_out;         /* [npoints] dJ_dv of the reference (= d loglik / d c),
                               reference node order (SEM_F_ADJOINT) or NULL           */
  int32_t* status_out;      /* [1] per-solve status (SEM_OK / SEM_ERR_NONFINITE) or NULL */
} sem_solve_t;

/* Launch configuration (the autotuner's knobs). */
typedef struct {
  int32_t tile_ex, tile_ez;   /* tile kernel: elements per CTA tile in x and z; 0 x 0 =
                                 automatic (of 8x8 .. 2x1 the finest whose CTAs over
                                 the batch are all resident at once, else 8x8)      */
  int32_t threads;            /* tile kernel: threads per CTA (multiple of 32, <= 256) */
  int32_t graph_chunk;        /* ticks per captured CUDA graph; 0 = plain launches    */
  int32_t kernel;             /* 0 auto, 1 tile kernel (one CTA per element tile),
                                 2 strip kernel (one CTA per full-height strip, TMA-
                                 staged element-row bands), 3 persistent tile kernel
                                 (the tile kernel's ticks in one cooperative launch with
                                 a grid barrier between ticks, for one-order groups
                                 whose tiles are all resident at once; otherwise the
                                 tile kernel per tick), 4 persistent strip kernel (the
                                 strip kernel's ticks in one cooperative launch, each CTA
                                 waiting only for its four neighbours' previous tick, for
                                 one-order groups whose chunks are all resident at once;
                                 otherwise the strip kernel per tick); auto picks strips
                                 when the batch has at least one strip per SM            */
  int32_t strip_bands;        /* strip kernel: element rows per CTA; 0 = automatic
                                 (full-height strips when the batch's strips give 2
                                 CTAs per SM, else chunks of >= 4 rows so that strips
                                 x chunks comes near 4 per SM; a chunk recomputes the
                                 z-line segments of the element row above it)        */
  int64_t memory_budget;      /* device bytes the workspaces of solves with ckpt_k = 0
                                 may use; 0 = 85% of (free + this batch's arena) less
                                 512 MiB.  Such batches run as consecutive groups, each
                                 with the largest checkpoint interval that fits (no
                                 replay when k = nt), the split chosen by a tick-cost
                                 model; results do not depend on the split            */
} sem_launch_cfg_t;

int sem_plan_create(const sem_plan_desc_t* desc, sem_plan_t** out);
int sem_plan_destroy(sem_plan_t* plan);
/* bytes of device workspace one solve of this plan needs with checkpoint interval k */
int64_t sem_plan_workspace_bytes(const sem_plan_t* plan, int32_t flags, int32_t ckpt_k);

int sem_batch_create(sem_batch_t** out);
int sem_batch_destroy(sem_batch_t* batch);
/* Run n solves (any mix of plans/orders/nt) to completion on ``stream``.  Solves of
 * the same polynomial order share one kernel launch per time tick.  cfg may be NULL:
 * every launch choice automatic (kernel, tile shape, strip chunks, memory budget). */
int sem_run(sem_batch_t* batch, const sem_solve_t* solves, int32_t n,
            const sem_launch_cfg_t* cfg, void* stream);
/* number of kernel launches issued by the last sem_run (for accounting) */
int64_t sem_batch_last_launches(const sem_batch_t* batch);
/* number of consecutive groups the last sem_run ran (1 unless ckpt_k = 0 solves were
 * split under the memory budget) */
int32_t sem_batch_last_groups(const sem_batch_t* batch);
/* launch shape the last sem_run used: tile kernel tile (elements) and strip kernel
 * element rows per CTA (0 when the tile kernel ran); any pointer may be NULL */
int sem_batch_last_shape(const sem_batch_t* batch, int32_t* tile_ex, int32_t* tile_ez,
                         int32_t* strip_bands);
/* tick rounds the last sem_run launched, summed over its groups (each round launches the
 * tick kernel once per polynomial order, then the tick counter kernel) */
int64_t sem_batch_last_ticks(const sem_batch_t* batch);
/* device time of the last sem_run's tick loops (CUDA events recorded on its stream
 * around each group's tick launches; set-up and output kernels excluded), in ms.
 * Waits for those events. */
int sem_batch_last_tick_ms(const sem_batch_t* batch, double* ms_out);
/* kernel variant used by the last sem_run: 1 tile, 2 strip, 3 persistent tile,
 * 4 persistent strip */
int32_t sem_batch_last_kernel(const sem_batch_t* batch);

/* Single-solve conveniences (plain path): forward with receivers in the run()
 * convention, and forward+adjoint in the run_forward_and_adjoint convention. */
int sem_forward(sem_batch_t* batch, const sem_plan_t* plan, const double* velocity,
                float* rec_out, void* stream);
int sem_forward_adjoint(sem_batch_t* batch, const sem_plan_t* plan, const double* velocity,
                        const double* y_obs, double inv_sigma2, int32_t exact,
                        int32_t ckpt_k, float* clean_out, double* loglik_out,
                        double* grad_out, void* stream);

/* Diagnostics (no counterpart in the reference): exercise the time limit of the device
 * waits without any fault.  which = 0: an mbarrier wait whose bytes never arrive (the
 * strip kernel's ring wait); 1: a grid barrier one arrival short (the persistent
 * kernel's tick barrier); 2: a grid barrier that completes.  Blocks about 2 s for
 * 0 and 1; *status_out = SEM_ERR_TIMEOUT for 0 and 1, SEM_OK for 2. */
int sem_selftest_wait(int32_t which, int32_t* status_out);

/* Allocation-free forward solve (receivers in the run() convention), for callers that
 * cannot allocate device memory while they run: a caller inside a memory pool that owns
 * the whole device, a real-time loop that must not hit cudaMalloc's implicit device
 * synchronisation, or an embedding whose allocator is not the CUDA runtime's.
 * No counterpart in the reference (MUN allocates its history with torch on every call).
 *
 * It uses a fixed 32 MiB scratch array that lives in this library's device image, so it
 * calls no cudaMalloc/cudaFree and nothing that allocates.  Every GPU that loads the
 * library holds that array until the process exits.  The plan must already exist
 * (sem_plan_create allocates; do it at set-up).  Limit: 4 float fields of
 * pitch x (nelz*npol+1) floats (pitch = nxg rounded up to 32) plus the tile map and
 * receiver sums must fit in 32 MiB, about 1.9 million mesh nodes; larger meshes
 * return SEM_ERR_ARG with the required size in sem_last_error().
 *
 * sem_plan_create looks up the array's device address (cudaGetSymbolAddress) with
 * the plan's device current and keeps it in the plan, so this call looks up and loads
 * nothing.  All calls share the one array and it keeps the last call's contents (the
 * call clears what must start at zero): calls that overlap on the GPU, from different
 * streams or threads, race and give wrong results.  status_out (device, may be NULL)
 * receives SEM_OK or SEM_ERR_NONFINITE. */
int sem_forward_noalloc(const sem_plan_t* plan, const double* velocity, float* rec_out,
                        int32_t* status_out, void* stream);

/* ---------------------------------------------------------------------------------
 * Serving engine: continuous batching (no counterpart in the reference, whose
 * drivers call SEMSimulation one request at a time: MCMC.py:193-208,
 * RQS_Coupling.py:295-351).  Solves are queued with sem_engine_submit and admitted at
 * the next tick boundary when a slot and enough device memory (the solve's workspace
 * under memory_cap) are free; each sem_engine_step retires finished solves, admits
 * queued ones and launches ticks_per_step ticks on the stream.  A solve's results do
 * not depend on what runs beside it (bitwise).  One thread uses an engine at a time.
 * ------------------------------------------------------------------------------- */
typedef struct sem_engine_s sem_engine_t;
typedef struct {
  int32_t max_solves;      /* concurrent solves                                        */
  int64_t memory_cap;      /* device bytes for solve workspaces (allocated at creation) */
  int32_t ticks_per_step;  /* ticks launched by one sem_engine_step                    */
  int32_t kernel;          /* 0 automatic per step (as in sem_run), 1 tile kernel,
                              2 strip kernel                                           */
  int32_t tile_ex, tile_ez;/* tile kernel tile size; 0 x 0 = automatic per step        */
} sem_engine_cfg_t;

int sem_engine_create(const sem_engine_cfg_t* cfg, sem_engine_t** out);
int sem_engine_destroy(sem_engine_t* engine);
/* queue one solve (same fields as in sem_run; its buffers must stay valid until it is
 * released) and return a ticket */
int sem_engine_submit(sem_engine_t* engine, const sem_solve_t* solve, int64_t* ticket);
/* retire, admit, launch ticks_per_step ticks */
int sem_engine_step(sem_engine_t* engine, void* stream);
/* *state: 0 queued, 1 running, 2 done (outputs written), -1 unknown ticket */
int sem_engine_status(sem_engine_t* engine, int64_t ticket, int32_t* state);
/* forget a done solve */
int sem_engine_release(sem_engine_t* engine, int64_t ticket);
/* out[5]: queued, running, workspace bytes in use, ticks launched, kernel launches */
int sem_engine_stats(const sem_engine_t* engine, int64_t* out);

/* ---------------------------------------------------------------------------------
 * Velocity model from a closed cubic B-spline interface (replaces
 * build_velocity_on_sem_nodes / build_velocity_layered_with_anomaly /
 * build_velocity_2d_background_with_anomaly: Bspline_Coupling/SEM/sem_waveform/
 * velocity.py:37-202, layered velocity.py:38-267, gridded velocity.py:54-332).
 * Per node: nearest curve sample, Newton refinement of the closest parameter, signed
 * distance (even-odd sign against the sample polygon), sigmoid or hard blend.
 * ------------------------------------------------------------------------------- */
typedef struct {
  int32_t ncoef;             /* coefficients of the closed curve (free points + 3)   */
  const double* knots;       /* HOST [ncoef + 4]                                     */
  const double* coef;        /* HOST [ncoef * 2] (x, z) pairs                        */
  double u_lo, u_hi;         /* valid parameter interval                             */
  int32_t nsamples;          /* initial-guess samples (<= 4096)                      */
  const double* u0;          /* DEVICE [nsamples] sample parameters                  */
  const double* samples;     /* DEVICE [nsamples * 2] C(u0), also the sign polygon    */
  int32_t newton_steps;
  double tau;                /* sigmoid width                                        */
  double v_inside;           /* velocity inside the curve                            */
  int32_t blend_replace;     /* 0: v_bg + (v_in - v_bg) sigmoid(-sd/tau); 1: v_in inside */
} sem_curve_t;

/* coords: DEVICE [npoints * 2]; v_background: DEVICE [npoints] or NULL (then v_outside);
 * outputs DEVICE: velocity [npoints], optional sd [npoints], u_star [npoints],
 * normal_out [npoints * 2] */
int sem_velocity_from_curve(const sem_curve_t* curve, int32_t npoints, const double* coords,
                            const double* v_background, double v_outside, double* velocity_out,
                            double* sd_out, double* ustar_out, double* normal_out, void* stream);
const char* sem_velocity_last_error(void);

/* Gradient of the log-likelihood w.r.t. the curve's K free control points for a batch
 * of S samples on one mesh, from dL/dv at the nodes (MUN's
 * _analytical_gradient_projection_improved, Bspline_Coupling/SEM/sem_waveform/core.py:902-970,
 * CO2_plume/layered_model/inversion/sem_waveform/core.py:1047-1117,
 * CO2_plume/one_stage/single_cubic/sem_waveform/core.py:1128-1202):
 *   sum over nodes with |dv| above the reference's threshold of
 *   dL/dv * (v_in - v_bg) sig (1 - sig) (-1/tau) * basis_j(u*) * outward normal.
 * knots: HOST [ncoef + 4] of the closed cubic spline (ncoef = K + 3: the clamped closure
 * repeats the first point 3 times, the periodic one the first 3 points; both fold back).
 * periodic != 0 applies the gridded package's parameter mapping lo + mod(u, 1) (hi - lo).
 * DEVICE inputs, row s = sample s: dL_dv, sd, ustar [S * npoints], normal [S * npoints * 2];
 * v_background DEVICE [npoints] or NULL (then v_background_const).  floor_one: threshold
 * 1e-8 * max(1, |v_in - v_bg|) (layered, gridded) instead of 1e-8 * |v_in - v_bg| (canonical).
 * grad_out DEVICE [S * 2K]: per sample K x-components, then K z-components.  Deterministic. */
int sem_project_from_curve(const double* knots, int32_t ncoef, int32_t K, int32_t periodic,
                           int32_t nsamples, int32_t npoints, const double* dL_dv, const double* sd,
                           const double* ustar, const double* normal, const double* v_background,
                           double v_background_const, double v_inside, double tau, int32_t floor_one,
                           double* grad_out, void* stream);

/* last error message of the calling thread (static storage) */
const char* sem_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
