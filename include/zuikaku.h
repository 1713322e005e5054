/* zuikaku.h -- C ABI of the B200 (sm_100a) per-step compute for ZuikakuCFD's
 * explicit 2D Euler solvers: WENO5 finite volume and DG P=1..3, SSP-RK3, the
 * DG limiters and the CFL max-wavespeed reduction.
 *
 * Every entry point returns an int status (ZK_OK = 0) and never throws.  A
 * context owns its device state and one CUDA stream; it is externally
 * synchronised (one host thread at a time).  zk_last_error() gives the message
 * of the last failure on the calling thread.
 *
 * Host arrays at this boundary are row-major planes, row i = y index (row 0 on
 * top, as in the reference's .dat files), column j = x:
 *   WENO state   double U[4][ny][nx]          rho, rho*u, rho*v, E
 *   DG state     double dof[4][NM][ny][nx]    NM = (P+1)^2, mode m = px*(P+1)+py
 *   bctype       int32 [ny][nx]               0 fluid, -1 copy ghost, 1 slip
 *                                             wall (DG), -3 exchange ghost
 * The reference stores the same fields as column-major Eigen matrices
 * (src_WENO/fluid.h:26-80, src_DG/fluid.h:44-110); src_WENO/fluid.cpp:391-393
 * gives its index map idx(i,j) = j*ny + i.
 */
#ifndef ZUIKAKU_H
#define ZUIKAKU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
    ZK_OK = 0,
    ZK_ERR_ARG = 1,       /* invalid argument (null pointer, bad size, bad option) */
    ZK_ERR_STATE = 2,     /* call out of order (no mesh set, ...)                  */
    ZK_ERR_CUDA = 3,      /* a CUDA runtime call failed                            */
    ZK_ERR_NUMERIC = 4,   /* the device status word reported NaN / non-positive    */
    ZK_ERR_UNSUPPORTED = 5,
    ZK_ERR_IO = 6,
    ZK_ERR_TIMEOUT = 7
};

/* ---- options -------------------------------------------------------------- */
enum { ZK_METHOD_WENO = 0, ZK_METHOD_DG = 1 };
/* FP64: the reference's arithmetic op for op (bit-identical to the reference
 * built with -ffp-contract=off).  MIXED: FP32 reconstruction/fluxes/quadrature
 * with FP64 conserved-state accumulation and FP64 pressure recovery.
 * FP64_FMA: FP64 throughout with multiply-adds fused, as the reference's own
 * Makefile build contracts them (within 1e-10 of that build, not bit-identical;
 * single contexts only, not the batched runner); DG stages run as one fused,
 * sum-factorised kernel per stage, the FP64 twin of the mixed-precision one. */
enum { ZK_PREC_FP64 = 0, ZK_PREC_MIXED = 1, ZK_PREC_FP64_FMA = 2 };
/* DG limiter: REFERENCE = Persson modal filter + Zhang-Shu positivity
 * (src_DG/fluid.cpp:824-992); NONE; TVB = Cockburn-Shu TVB minmod (M) with
 * characteristic limiting; TVB_MLP = TVB limiting of the cells a learned
 * indicator flags. */
enum { ZK_LIMITER_REFERENCE = 0, ZK_LIMITER_NONE = 1, ZK_LIMITER_TVB = 2, ZK_LIMITER_TVB_MLP = 3 };
enum { ZK_FLUX_HLLC = 0, ZK_FLUX_HLL = 1 };
/* Boundary handling of bctype -3 cells: EXCHANGE leaves them alone (the
 * reference at one rank); PERIODIC refills them with their periodic image
 * inside the 3-wide ring before every RHS evaluation. */
enum { ZK_BOUNDARY_EXCHANGE = 0, ZK_BOUNDARY_PERIODIC = 1 };
/* WENO face reconstruction: WENO5 (the reference's scheme,
 * src_WENO/fluid.cpp:230-263) or MUSCL with the slope limiter of the
 * reference's muscl_reconstruct (src_WENO/fluid.cpp:203-225, which its solver
 * never calls): minmod, van Leer, superbee.  MUSCL runs at FP64 and FP64_FMA
 * precision on single contexts. */
enum { ZK_RECON_WENO5 = 0, ZK_RECON_MUSCL_MINMOD = 1, ZK_RECON_MUSCL_VANLEER = 2, ZK_RECON_MUSCL_SUPERBEE = 3 };

typedef struct zk_options {
    int method;     /* ZK_METHOD_*                           */
    int order;      /* DG polynomial degree P in 1..3        */
    int precision;  /* ZK_PREC_*                             */
    int limiter;    /* ZK_LIMITER_* (DG only)                */
    int flux;       /* ZK_FLUX_* (DG only; WENO is HLLC)     */
    int boundary;   /* ZK_BOUNDARY_*                         */
    int device;     /* CUDA device ordinal                   */
    double tvb_M;   /* TVB constant M (default 50)           */
    int recon;      /* ZK_RECON_* (WENO only; default WENO5) */
    int tile_tpc;   /* mixed DG: threads per cell of the stage kernel, 1 or 2;
                       0 (default) = chosen by timing both on the first step */
} zk_options;

typedef struct zk_ctx zk_ctx;

/* Fills *opt with defaults: WENO, P=2, FP64, reference limiter, HLLC,
 * exchange boundary, device 0, M=50, WENO5 reconstruction. */
void zk_default_options(zk_options* opt);

int zk_create(const zk_options* opt, zk_ctx** out);
int zk_destroy(zk_ctx* ctx);
const char* zk_last_error(void);
int zk_version(void);

/* Grid and boundary codes; allocates the device state.  Replaces the sizing
 * part of Mesh(folder) (src_WENO/fluid.cpp:68-94, src_DG/fluid.cpp:216-244). */
int zk_set_mesh(zk_ctx* ctx, int ny, int nx, double da, double gamma, const int32_t* bctype);

/* Host <-> device state (layouts above).  The state stays device-resident
 * between steps; these are the only host copies the step loop needs. */
int zk_set_state(zk_ctx* ctx, const double* host_state);
int zk_get_state(zk_ctx* ctx, double* host_state);
/* Number of doubles in the host state (4*ny*nx or 4*NM*ny*nx). */
size_t zk_state_size(const zk_ctx* ctx);

/* Mesh(folder): read params.txt + rho/u/v/p/bctype.dat, convert to conserved
 * variables and, for DG, initialise mode 0 (src_DG/fluid.cpp:173-182). */
int zk_load_case(zk_ctx* ctx, const char* dir);

/* updateMesh x nsteps: one SSP-RK3 step each (src_WENO/fluid.cpp:468-493,
 * src_DG/fluid.cpp:1005-1054), ghost fill and limiter included, fixed dt. */
int zk_step(zk_ctx* ctx, double dt, int nsteps);

/* computeRHS (src_WENO/fluid.cpp:328-463 / src_DG/fluid.cpp:656-807): fills
 * the ghosts of the device state in place, as the reference mutates its Mesh,
 * and writes dU to host memory.  WENO dU includes dt; DG dU = d(dof)/dt. */
int zk_rhs(zk_ctx* ctx, double dt, double* host_dU);

/* applyLimiter (src_DG/fluid.cpp:824-992) on the device state (DG only). */
int zk_limit(zk_ctx* ctx);

/* Max wave speed: WENO computeMaxSpeed (src_WENO/fluid.cpp:539-553, all
 * cells); DG computeMaxSpeedDG_omp (src_DG/solver.cpp:26-64, fluid cells,
 * 4 corners). */
int zk_max_speed(zk_ctx* ctx, double* out);

/* recoverPrimitives (src_WENO/fluid.cpp:500-515): prim[4][ny][nx] =
 * rho, u, v, p of the cell averages, FP64. */
int zk_recover_primitives(zk_ctx* ctx, double* host_prim);

/* Mach number mach[ny][nx] = |u| / sqrt(gamma p / rho) and speed[ny][nx] =
 * |u| (may be NULL) of the cell averages, computed on the device (the plot
 * notebook's compute_mach, plot.ipynb cell 0; no counterpart in the solver). */
int zk_mach_number(zk_ctx* ctx, double* host_mach, double* host_speed);

/* Device status word (bit 0: NaN seen, bit 1: rho <= 0, bit 2: p <= 0) of the
 * last zk_step, or of the zk_stage calls since the last stage 1; cleared by
 * each zk_step and each zk_stage(ctx, dt, 1). */
int zk_status_word(zk_ctx* ctx, uint32_t* out);

/* Stream control: run on an external stream (e.g. one owned by a framework)
 * instead of the context's own; NULL restores the context stream. */
int zk_set_stream(zk_ctx* ctx, void* cuda_stream);
int zk_synchronize(zk_ctx* ctx);

/* Timing helper: runs nsteps steps and returns the device time measured with
 * CUDA events on the context's stream. */
int zk_step_timed(zk_ctx* ctx, double dt, int nsteps, float* ms);

/* Threads per cell the mixed DG stage kernel of this context runs (1 or 2;
 * 0 before the first step).  No counterpart in the reference. */
int zk_tile_tpc(zk_ctx* ctx, int* tpc);

/* Device pointer of the FP64 state (layout: planes of ny rows x pitch
 * doubles) and its row pitch in elements, for zero-copy callers. */
int zk_state_device(zk_ctx* ctx, double** dptr, int* pitch);

/* ---- x-slab decomposition ----------------------------------------------------
 * A grid split into x-slabs, one context (and one GPU) each, as the
 * reference's MPI runs split it (splitMeshVertically, src_WENO/fluid.cpp:99-152):
 * every inner slab side carries 3 exchange columns (bctype -3, boundary
 * ZK_BOUNDARY_EXCHANGE), which a stage reads as stored and never updates.
 * One step of a slab is, for stage = 1, 2, 3:
 *   zk_stage(stage); [DG TVB limiters: exchange(stage); zk_stage_limit(stage);]
 *   exchange(stage)
 * where exchange(stage) sends the 3 owned columns next to each inner side to
 * the neighbour and stores the 3 columns received in the exchange columns --
 * exchangeConservativeColumns after every stage and limiter pass
 * (src_WENO/fluid.cpp:160-198, 468-493; src_DG/fluid.cpp:342-400, 1005-1054).
 * The owned cells of the slabs then hold the bits one context over the whole
 * grid computes.  All of these only enqueue work on the context's stream. */
/* Stage 1, 2 or 3 of one zk_step (the same kernels; the DG reference limiter
 * is part of the stage).  Stage 1 clears the status word and the limited-cell
 * count, as zk_step does. */
int zk_stage(zk_ctx* ctx, double dt, int stage);
/* The TVB pass zk_step runs after `stage` (DG TVB limiters; no-op otherwise). */
int zk_stage_limit(zk_ctx* ctx, int stage);
/* Halo of the state written by `stage` (0 or 3: U^n; 1, 2: the stage states):
 * nplanes x ny x 3 elements (FP32 for the stage states of a mixed-precision
 * DG context, else FP64), buffer layout [plane][row][column].  side 0 = left,
 * 1 = right.  zk_halo_pack copies the 3 owned columns next to that side
 * (3..5, or nx-6..nx-4) into dev_buf; zk_halo_unpack copies dev_buf into the
 * exchange columns of that side (0..2, or nx-3..nx-1).  dev_buf is device
 * memory of at least zk_halo_bytes bytes on the context's device. */
int zk_halo_bytes(zk_ctx* ctx, int stage, size_t* bytes);
int zk_halo_pack(zk_ctx* ctx, int stage, int side, void* dev_buf);
int zk_halo_unpack(zk_ctx* ctx, int stage, int side, const void* dev_buf);

/* ---- learned troubled-cell indicator (no counterpart in the reference) ----
 * A 40 -> 32 -> 32 -> 32 -> 1 GELU MLP gates the TVB limiter of
 * ZK_LIMITER_TVB_MLP contexts: only cells with a positive logit take the
 * characteristic-limiting branch.  Its inputs for the output of an RK stage
 * are the cell's rho and E modes in that output and the cell's and its
 * neighbours' means in the stage's INPUT.  Mixed-precision P=2/3 contexts
 * evaluate it inside the stage kernel on the tensor cores (BF16) and limit
 * only the cells it lists; other contexts run a gated pass after each stage.
 * Parameters are the flat FP32 block w1[32][40], b1[32], w2[32][32], b2[32],
 * w3[32][32], b3[32], w4[32], b4 (ZK_MLP_NPARAM floats), rounded to BF16 for
 * inference. */
#define ZK_MLP_NPARAM 3457
#define ZK_MLP_IN 40
int zk_set_indicator(zk_ctx* ctx, const float* params, int nparams);
/* The indicator's screen: a cell whose 40 features all lie within `screen` of
 * a constant state's (all 0) is smooth without evaluating the network, and a group of cells evaluated
 * together (a warp) that is all smooth skips it.  The trained weights come
 * with a screen calibrated to keep every TVB-troubled training cell; < 0
 * (the default) evaluates every cell. */
int zk_set_indicator_screen(zk_ctx* ctx, float screen);
/* Per cell of the current (FP64) state: the indicator's 40 input features
 * with the state's own means (features[ny*nx][40], may be NULL) and the plain
 * TVB troubled-cell flag (labels[ny][nx], may be NULL).  The state is not
 * modified. */
int zk_indicator_features(zk_ctx* ctx, float* features, uint8_t* labels);
/* The logits[ny*nx] of the gated pass for the current state with its own
 * means (0 for non-updated cells). */
int zk_indicator_logits(zk_ctx* ctx, float* logits);
/* After zk_stage(ctx, dt, stage): per cell of that stage's output, the
 * indicator's 40 features (its modes, the stage input's means;
 * features[ny*nx][40], may be NULL) and the plain TVB flag of the output
 * (labels[ny][nx], may be NULL) -- the training data of the indicator. */
int zk_indicator_stage_features(zk_ctx* ctx, int stage, float* features, uint8_t* labels);
/* zk_stage(ctx, dt, stage) of a mixed-precision DG P=2/3 TVB_MLP context,
 * returning per cell the features and logit the fused stage kernel computed
 * (features[ny*nx][40], logits[ny*nx], either may be NULL; 0 for cells not
 * updated) and the number of cells it listed for limiting (may be NULL). */
int zk_indicator_stage_logits(zk_ctx* ctx, double dt, int stage, float* features, float* logits,
                              uint32_t* listed);
/* Cells the TVB passes limited during the last zk_step (summed over stages). */
int zk_limited_cells(zk_ctx* ctx, uint32_t* count);
/* Training on the GPU (hand-written FP32 forward/backward + Adam kernels):
 * X[n][40] features, y[n] labels (0/1); params in = initial, out = trained;
 * batch a multiple of 64; loss = BCE on the logit with positive weight. */
int zk_mlp_train(int device, const float* X, const uint8_t* y, int64_t n, float* params, int epochs, int batch,
                 float lr, float pos_weight, uint64_t seed, float* epoch_loss);
/* Mean loss and mean parameter gradient over n samples (gradient checks). */
int zk_mlp_grad(int device, const float* X, const uint8_t* y, int64_t n, const float* params, float pos_weight,
                float* grad, float* loss);
/* Logits of n samples (bf16 != 0: BF16-rounded weights, as in inference). */
int zk_mlp_forward(int device, const float* X, int64_t n, const float* params, int bf16, float* logits);

/* Failure-detection self-test (no counterpart in the reference): runs stage 1
 * of a mixed-precision WENO context with its TMA barrier expecting 16 bytes
 * more than the copy delivers and its bounded wait limited to spin_limit polls
 * (0: 1), so every CTA's wait runs out; each CTA records STATUS_TIMEOUT (8) in
 * the status word, settles the missing bytes, waits for its copy to land and
 * leaves without writing.  *status_out receives the status word; the state is
 * untouched and the context stays usable.  No GPU fault is involved. */
int zk_selftest_tma_timeout(zk_ctx* ctx, uint32_t spin_limit, uint32_t* status_out);

/* FMA-throughput microbenchmark of one device: kind 0 = FP64, 1 = FP32;
 * writes the achieved dense TFLOP/s (2 flops per FMA).  Roofline denominator
 * for kernels bound by the FP pipes. */
int zk_peak_flops(int device, int kind, double* tflops);

/* No counterpart in the reference.  The FP64 WENO5 SSP-RK3 step of zk_step
 * (same kernels, bit-identical results) for callers that cannot allocate GPU
 * memory: applications whose device memory is owned by another allocator (a
 * framework's caching allocator or a pool reserved at start-up) and loops
 * that must not pay cudaMalloc's implicit synchronisation.  The caller passes
 * device pointers to the state (planes of ny rows x pitch doubles, updated in
 * place) and to bctype (int32 [ny][nx]); the stage states, ghost map and
 * status word live in a fixed scratch array inside the library (about
 * 17.3 MiB held on each GPU that loads it, until exit).  Limit:
 * ny * pitch <= 262144 cells, else ZK_ERR_ARG.  Runs on `stream` (NULL = the
 * default stream) of the current device.  The first call on a device looks up
 * the scratch address and must come before any stream capture; so must the
 * first call after that device's context was reset (cudaDeviceReset), which
 * looks it up again.  Calls whose
 * GPU work overlaps race on the shared scratch.  status_out (host, may be
 * NULL) receives the status word and makes the call synchronous. */
int zk_weno_step_noalloc(double* state, int ny, int nx, int pitch, double da, double gamma,
                         const int32_t* bctype, double dt, int nsteps, void* stream,
                         uint32_t* status_out);

/* ---- batched runner --------------------------------------------------------
 * No counterpart in the reference, whose solver.cpp advances one mesh per
 * process (src_WENO/solver.cpp:159-190, src_DG/solver.cpp:270-310).  A batch
 * holds many independent problems of any sizes, WENO and DG mixed, each with
 * its own step count and CFL number, and advances them on one GPU:
 *   - problems with the same method, precision and order form a group; each RK
 *     stage of a group is ONE persistent kernel launch over the tiles of all
 *     its running problems (a device-side directory lists them);
 *   - each step is max wave speed -> per-problem dt -> 3 stages -> step count,
 *     all on the device (dt never goes through the host); graph_steps steps
 *     of every group are captured once as a CUDA graph and replayed;
 *   - an autotuner times the tile variants and persistent grid sizes of each
 *     group's stage kernel before the first run;
 *   - the scheduler admits all problems at once (ZK_BATCH_ALL) or
 *     smallest-work-first while the running problems hold fewer than
 *     active_cells updated cells (ZK_BATCH_SJF), refilling as problems finish.
 * A problem's dt: WENO cfl*da/lambda (lambda = computeMaxSpeed of the step's
 * input, src_WENO/fluid.cpp:539-553); DG cfl*dgSafeDt(lambda)
 * (src_DG/solver.cpp:19-64).  DG limiters: REFERENCE or NONE. */
typedef struct zk_batch zk_batch;

enum { ZK_BATCH_ALL = 0, ZK_BATCH_SJF = 1 };
enum { ZK_BATCH_WAITING = 0, ZK_BATCH_RUNNING = 1, ZK_BATCH_DONE = 2, ZK_BATCH_FAILED = 3 };

typedef struct zk_batch_options {
    int device;
    int policy;           /* ZK_BATCH_*                                            */
    double active_cells;  /* SJF admission bound in updated cells (<= 0: 8e6)      */
    int graph_steps;      /* RK steps per captured graph (1..1000; default 10)     */
    int autotune;         /* 0 off, 1 on (cached per process), 2 re-tune           */
    size_t arena_bytes;   /* > 0: one device allocation all problems carve from    */
    int weno_variant;     /* -1: tuned; 0..5: pin the WENO tile variant (the      */
                          /* autotuner then tunes CTAs per SM only)               */
    int dg_variant;       /* -1: tuned; 0..3: pin the mixed DG tile variant       */
} zk_batch_options;

typedef struct zk_batch_report {
    double ms;              /* device time of the run (CUDA events)               */
    double cell_updates;    /* sum over problems of updated cells x steps taken   */
    double dof_updates;     /* the same x DOF per cell (4, or 4 (P+1)^2 for DG)   */
    double latency_p50_ms;  /* per-problem completion time from the run's start   */
    double latency_p99_ms;
    double latency_max_ms;
    int problems, done, failed;
    int graph_launches, graph_steps;
    long long kernel_launches; /* kernels the replayed graphs launched            */
} zk_batch_report;

typedef struct zk_batch_problem {
    int state;          /* ZK_BATCH_*                                  */
    int steps_done;
    double t;           /* simulated time reached                      */
    double latency_ms;  /* completion time from the run's start, or -1 */
    uint32_t status;    /* status word bits of this problem's kernels  */
    int group;
} zk_batch_problem;

void zk_batch_default_options(zk_batch_options* o);
int zk_batch_create(const zk_batch_options* o, zk_batch** out);
/* Register one problem: options as for zk_create, mesh as for zk_set_mesh,
 * initial state as for zk_set_state (host layout above).  *id = 0, 1, ... */
int zk_batch_add(zk_batch* b, const zk_options* opt, int ny, int nx, double da, double gamma,
                 const int32_t* bctype, const double* state, int nsteps, double cfl, int* id);
/* Advance every problem to its step count (once per batch). */
int zk_batch_run(zk_batch* b, zk_batch_report* report);
int zk_batch_get_state(zk_batch* b, int id, double* host);
int zk_batch_problem_info(zk_batch* b, int id, zk_batch_problem* out);
/* The dt of each step problem `id` took (n <= its step count). */
int zk_batch_dt_history(zk_batch* b, int id, double* dts, int n);
/* Chosen configuration of group g (groups form at zk_batch_run): tile variant
 * of the stage kernel (WENO: 3 * h + k, tile height {4, 8}[h] worked by
 * {rows/2 + 1, rows + 1, 2 rows + 2}[k] warps; mixed DG: 2 * t + h, tile
 * height {2, 4}[h] at t + 1 threads per cell) and its CTAs per SM; *ngroups =
 * number of groups.  Any pointer may be NULL; g = -1 only reports the number
 * of groups. */
int zk_batch_group_config(zk_batch* b, int g, int* method, int* precision, int* order, int* variant,
                          int* ctas_per_sm, int* ngroups);
/* Tile of group g's stage kernel: cells per tile (tile_rows x tile_cols) and
 * the threads that work one tile, so threads per cell = threads_per_tile /
 * (tile_rows * tile_cols).  Any pointer may be NULL. */
int zk_batch_group_tile(zk_batch* b, int g, int* tile_rows, int* tile_cols, int* threads_per_tile);
void zk_batch_destroy(zk_batch* b);

#ifdef __cplusplus
}
#endif
#endif
