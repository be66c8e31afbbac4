/*
 * tse_cuda.h -- C-ABI of libtsecuda.so, the sm_100a implementation of the
 * TRANSPORTSE time-step core.
 *
 * The reference (thkempka/transportse, tse.py) has no foreign-function
 * interface: its kernels are numba functions called from the Python driver
 * loop.  Each entry point below replaces one of those functions, keeps its
 * argument meaning and its return values, and is called from the Python
 * driver (transportse_b200.driver) through ctypes.
 *
 * Conventions
 *  - All array pointers are DEVICE pointers to C-order (nx, ny, nz) float64
 *    arrays (k fastest), the layout of tse.py:81-157.  Species fields are
 *    passed one species at a time as contiguous (nx, ny, nz) arrays.
 *  - The caller owns every buffer.  Entry points that need scratch take a
 *    caller-provided device workspace whose size is returned by
 *    tse_workspace_bytes(); nothing allocates on the hot path.
 *  - Every call is stream-ordered on the given stream (a cudaStream_t passed
 *    as void*; NULL = legacy default stream) and returns before the work
 *    completes.  Solver results go to a device-resident TseSolveStatus,
 *    readable after the stream is synchronised.
 *  - Return value: TSE_OK, or a negative TSE_ERR_* code for invalid
 *    arguments, a too-small workspace or a failed launch.
 *  - Bounded waits: the persistent solver kernels synchronise their blocks
 *    with a grid barrier whose wait is bounded in time; on timeout they set
 *    TseSolveStatus.error = TSE_STATUS_BARRIER_TIMEOUT and return.
 *  - Re-entrant across streams when each stream has its own workspace and
 *    status buffers.
 */
#ifndef TSE_CUDA_H
#define TSE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSE_OK 0
#define TSE_ERR_ARG (-1)
#define TSE_ERR_WORKSPACE (-2)
#define TSE_ERR_LAUNCH (-3)
#define TSE_ERR_DEVICE (-4)

#define TSE_STATUS_OK 0
#define TSE_STATUS_BARRIER_TIMEOUT 1

/* Grid geometry: the module-level globals dx, dy, dz, g and beta that the
 * reference kernels read (tse.py:82-96).  sin_beta / cos_beta are
 * numpy.sin(beta) / numpy.cos(beta) evaluated on the host. */
typedef struct TseGrid {
    int32_t nx, ny, nz, reserved;
    const double *dx, *dy, *dz; /* device, lengths nx, ny, nz */
    double g, sin_beta, cos_beta;
} TseGrid;

/* Result of one solver call: the tuple the reference functions return
 * (t, dt, converged, num_it) plus diagnostics.  Up to 8 dt-halving events
 * (iteration, dt before halving, L2 at that iteration) are recorded for the
 * log lines of tse.py:730-732, 902-904, 1070-1071. */
typedef struct TseSolveStatus {
    double t;          /* t_P / t_C / t_T: accumulated dt of the solve */
    double dt;         /* dt_P / dt_C / dt_T: next time-step size */
    double diff;       /* last relative L2 change */
    int32_t converged;
    int32_t num_it;
    int32_t num_sub_it;
    int32_t halvings;
    int32_t error;     /* TSE_STATUS_* */
    int32_t n_events;
    int32_t ev_it[8];
    double ev_dt[8];
    double ev_diff[8];
    int32_t cycles;    /* mixed-precision forms: FP64 residual evaluations */
    int32_t reserved;
} TseSolveStatus;

/* Pressure solve arguments, compute_P(P, c_f, nue, rho_f, phi, Kx, Ky, Kz,
 * qx, qy, qz, dt_P, BP, WP, SOR, max_it, inc_it, max_dt, min_dt, P_conv)
 * (tse.py:647-650).  qx/qy/qz are not read by the reference solve and are
 * omitted.  c_r is the compressibility array numba froze at first call. */
typedef struct TsePressureArgs {
    double *P;        /* in/out */
    double *Pn;       /* out: P at entry (the returned Pn) */
    const double *c_f, *nue, *rho_f, *phi, *Kx, *Ky, *Kz, *c_r, *BP, *WP;
    double dt_P, SOR, inc_it, max_dt, min_dt, P_conv;
    int32_t max_it;
    int32_t sweep;    /* FP64 solves' sweep kernel for this call (no counterpart
                         in the reference): 0 the bulk-copy staged kernel
                         wherever its stages fit, else plain loads (default);
                         1 plain loads.  Same cell values either way.  The
                         mixed-precision forms ignore it. */
} TsePressureArgs;

/* Species transport arguments, compute_C(C, D_fx, D_fy, D_fz, phi, rho_f,
 * qx, qy, qz, dt_C, BC, WC, RC, e, omega, SOR, max_it, inc_it, max_dt,
 * min_dt, C_conv) (tse.py:783-786); l_l / l_t are the frozen lf_l / lf_t
 * and imblflo the frozen config.C_IMBLFLO. */
typedef struct TseSpeciesArgs {
    double *C;        /* in/out, one species */
    const double *D_fx, *D_fy, *D_fz, *phi, *rho_f, *qx, *qy, *qz, *BC, *WC, *RC, *e;
    const double *l_l, *l_t;
    double dt, omega, SOR, inc_it, max_dt, min_dt, conv;
    int32_t max_it, imblflo;
    int32_t sweep;    /* as TsePressureArgs.sweep */
    int32_t reserved;
} TseSpeciesArgs;

/* Heat transport arguments, compute_T(T, l_f, cp_f, rho_f, phi, qx, qy, qz,
 * dt_T, BT, WT, e, omega, SOR, max_it, inc_it, max_dt, min_dt, T_conv)
 * (tse.py:919-922); l_r / rho_r / cp_r / l_l / l_t are the frozen l_r,
 * rho_r, cp_r, lt_l, lt_t and imblflo the frozen config.T_IMBLFLO. */
typedef struct TseHeatArgs {
    double *T;        /* in/out, one temperature layer */
    const double *l_f, *cp_f, *rho_f, *phi, *qx, *qy, *qz, *BT, *WT, *e;
    const double *l_r, *rho_r, *cp_r, *l_l, *l_t;
    double dt, omega, SOR, inc_it, max_dt, min_dt, conv;
    int32_t max_it, imblflo;
    int32_t sweep;    /* as TsePressureArgs.sweep */
    int32_t reserved;
} TseHeatArgs;

/* Workspace kinds for tse_workspace_bytes(). */
#define TSE_WS_PRESSURE 1
#define TSE_WS_TRANSPORT 2
#define TSE_WS_REDUCE 3
#define TSE_WS_PRESSURE_DC 4
#define TSE_WS_TRANSPORT_DC 5

/* Bytes of device workspace a call of the given kind needs for this grid. */
size_t tse_workspace_bytes(const TseGrid *grid, int32_t kind);

/* Red-black SOR pressure solve with the convergence / dt-halving loop of
 * compute_P (tse.py:647-742), FP64, reference operation order.  Replaces
 * tse.py:647. */
int32_t tse_compute_P(const TseGrid *grid, const TsePressureArgs *args,
                      TseSolveStatus *d_status, void *d_workspace,
                      size_t workspace_bytes, void *stream);

/* Mixed-precision forms of compute_P / compute_C / compute_T (tse.py:647,
 * 783, 919): the FP64 residual of the reference's per-cell equation drives
 * red-black SOR sweeps on an FP32 correction, which is added to the FP64
 * iterate every `cycle` iterations and at convergence.  Same arguments,
 * convergence test, dt control and results as the FP64 entry points;
 * agreement with them is to the solver tolerance, not bit for bit.  These
 * calls synchronise the stream once per correction cycle (they read the
 * sweep kernel's event record) and return when the solve is done.
 * Workspace: TSE_WS_PRESSURE_DC / TSE_WS_TRANSPORT_DC. */
typedef struct TseDcOptions {
    int32_t cycle;            /* in: iterations per correction cycle, <= 0: 256 */
    int32_t max_blocks;       /* in: cap on the sweep kernel's blocks, <= 0: as
                                 many as fit; lets several solves share the GPU */
    int32_t timing;           /* in: 1 = time the sweep-kernel launches (CUDA
                                 events on the call's stream; the global timer
                                 inside the device-driven loop's graph) */
    int32_t sweep_launches;   /* out (timing): sweep-kernel launches */
    int64_t sweep_iterations; /* out (timing): red+black iterations they ran */
    double sweep_ms;          /* out (timing): their summed event time */
    int32_t host_loop;        /* in, batched fused form only: 0 (default) the
                                 device-driven loop, one CUDA graph launch per
                                 call; 1 a host round trip per sweep launch.
                                 Same results bit for bit. */
    int32_t reserved;
    double loop_ms;           /* out (timing, batched fused form): event time of
                                 the whole loop around the sweeps (plan, sweeps,
                                 events, x += d, residuals); in the device-driven
                                 loop sweep_ms is then the sweep kernel's own
                                 time, taken with the device's global timer */
    int32_t chunk;            /* in/out, single-model forms: the staged sweep's
                                 chunk of cells (256, 512, 1024; else 512) --
                                 on return the variant that ran, 0 for the
                                 plain-load sweep (no stages fit) */
    int32_t ring;             /* in/out: stages a pipeline (2..4; else as many
                                 as fit, up to 4) */
    int32_t pipes;            /* in/out: pipelines a block (1: two blocks per
                                 SM; else 2: one block per SM) */
    int32_t graph_runs;       /* in/out, batched fused form, device-driven loop:
                                 loop-body runs per graph launch before the host
                                 relaunches the graph (<= 0: 4096); on return,
                                 the graph launches the call made */
    int64_t active_cells;     /* in, batched fused form with the device-driven
                                 loop: cells (both colours, padding included)
                                 solving at once; the items wait in index order
                                 and join as earlier ones finish (the first
                                 waiting item always when none runs); <= 0:
                                 every item from the start.  Each model's
                                 results are those of its solve alone either
                                 way. */
} TseDcOptions;
int32_t tse_compute_P_dc(const TseGrid *grid, const TsePressureArgs *args,
                         TseDcOptions *opts, TseSolveStatus *d_status,
                         void *d_workspace, size_t workspace_bytes,
                         void *stream);
int32_t tse_compute_C_dc(const TseGrid *grid, const TseSpeciesArgs *args,
                         TseDcOptions *opts, TseSolveStatus *d_status,
                         void *d_workspace, size_t workspace_bytes,
                         void *stream);
int32_t tse_compute_T_dc(const TseGrid *grid, const TseHeatArgs *args,
                         TseDcOptions *opts, TseSolveStatus *d_status,
                         void *d_workspace, size_t workspace_bytes,
                         void *stream);

/* Batched mixed-precision solves: the compute_P / compute_C / compute_T
 * calls of n independent models (an ensemble, or the requests a server is
 * stepping together).  Each item is exactly the single-model call of
 * tse_compute_*_dc -- its own grid, arguments, status record and workspace
 * (TSE_WS_PRESSURE_DC / TSE_WS_TRANSPORT_DC; no two items may share one) --
 * and gets the same results to the solver tolerance.  opts->cycle as for the
 * single-model form.  With opts->timing, the fused form writes the number of
 * its sweep launches, the global iterations they ran and their summed CUDA
 * event time (the cluster form writes nothing).
 *   opts->max_blocks <= 0: fused form -- every model's cells in one
 *     cooperative sweep sharing its barriers (models that finish drop out);
 *     the loop around the sweeps runs on the device as one CUDA graph launch
 *     (a conditional WHILE node whose body plans the launch, sweeps, handles
 *     each model's events and forms the residuals; the call reads one small
 *     record at the end) -- or, with opts->host_loop = 1 or on the legacy
 *     default stream, on the host, one stream synchronisation per sweep
 *     launch; the same results bit for bit; with opts->timing the device
 *     loop reports its whole time in sweep_ms; the call returns when every
 *     solve is done;
 *   opts->max_blocks > 0: cluster form -- one persistent launch with one
 *     thread-block cluster of max_blocks CTAs (at most 16) per model; the
 *     call returns after queueing the work, nothing is read back.
 * d_batch_ws holds tse_batch_workspace_bytes(n, total_cells) bytes, where
 * total_cells is the sum of nx*ny*nz over the items.  A non-finite dt or
 * min_dt is TSE_ERR_ARG.  Replaces n calls of tse.py:647 / 783 / 919. */
typedef struct TseBatchPressure {
    const TseGrid *grid;
    const TsePressureArgs *args;
    TseSolveStatus *d_status;
    void *d_workspace;
    size_t workspace_bytes;
} TseBatchPressure;
typedef struct TseBatchSpecies {
    const TseGrid *grid;
    const TseSpeciesArgs *args;
    TseSolveStatus *d_status;
    void *d_workspace;
    size_t workspace_bytes;
} TseBatchSpecies;
typedef struct TseBatchHeat {
    const TseGrid *grid;
    const TseHeatArgs *args;
    TseSolveStatus *d_status;
    void *d_workspace;
    size_t workspace_bytes;
} TseBatchHeat;
size_t tse_batch_workspace_bytes(int32_t n, int64_t total_cells);
int32_t tse_compute_P_dc_batch(const TseBatchPressure *items, int32_t n,
                               TseDcOptions *opts, void *d_batch_ws,
                               size_t batch_ws_bytes, void *stream);
int32_t tse_compute_C_dc_batch(const TseBatchSpecies *items, int32_t n,
                               TseDcOptions *opts, void *d_batch_ws,
                               size_t batch_ws_bytes, void *stream);
int32_t tse_compute_T_dc_batch(const TseBatchHeat *items, int32_t n,
                               TseDcOptions *opts, void *d_batch_ws,
                               size_t batch_ws_bytes, void *stream);

/* Pressure solve that allocates nothing and takes no workspace.  It has no
 * counterpart in the reference; it exists for callers that cannot allocate
 * device memory themselves -- a host program whose device memory belongs to
 * someone else's allocator and that can pass only its field buffers, or one
 * whose time loop must not stall on cudaMalloc, which can synchronise the
 * device.  Same arguments and results as tse_compute_P, except that the
 * scratch is a fixed TSE_NOALLOC_SCRATCH_BYTES (6 MiB) device array inside
 * the library, reserved on every GPU that loads it until the process exits.
 * That holds grids of up to about 43,000 cells (32 x 32 x 32 fits); larger
 * grids return TSE_ERR_WORKSPACE and launch nothing.  The first call on a
 * device looks up the array's device address, so make that first call before
 * any stream capture.  The address is kept for the life of the process, so
 * calls after a cudaDeviceReset (or any teardown of the device's primary
 * context) are not supported.  All calls on one GPU share the array: calls
 * that overlap on the GPU (other streams or host threads) race and must be
 * serialised by the caller. */
#define TSE_NOALLOC_SCRATCH_BYTES (6 * 1024 * 1024)
int32_t tse_compute_P_noalloc(const TseGrid *grid, const TsePressureArgs *args,
                              TseSolveStatus *d_status, void *stream);

/* Darcy face fluxes, compute_q (tse.py:744-780); the last plane of each
 * component is left untouched as in the reference.  Replaces tse.py:744. */
int32_t tse_compute_q(const TseGrid *grid, const double *P, const double *BP,
                      const double *Kx, const double *Ky, const double *Kz,
                      double *qx, double *qy, double *qz, const double *nue,
                      const double *rho_f, void *stream);

/* Local flow-balance error, flow_error (tse.py:409-446).  Replaces
 * tse.py:409. */
int32_t tse_flow_error(const TseGrid *grid, const double *P, const double *Pn,
                       const double *qx, const double *qy, const double *qz,
                       const double *WP, const double *phi, const double *c_f,
                       const double *c_r, const double *rho_f, double dt_P,
                       double *e, void *stream);

/* Species transport solve, compute_C (tse.py:783-916).  Replaces
 * tse.py:783. */
int32_t tse_compute_C(const TseGrid *grid, const TseSpeciesArgs *args,
                      TseSolveStatus *d_status, void *d_workspace,
                      size_t workspace_bytes, void *stream);

/* Heat transport solve, compute_T (tse.py:919-1081).  Replaces tse.py:919. */
int32_t tse_compute_T(const TseGrid *grid, const TseHeatArgs *args,
                      TseSolveStatus *d_status, void *d_workspace,
                      size_t workspace_bytes, void *stream);

/* Smolarkiewicz anti-diffusive velocities, smolarkiewicz (tse.py:1083-1116).
 * Replaces tse.py:1083. */
int32_t tse_smolarkiewicz(const TseGrid *grid, const double *C,
                          const double *qx, const double *qy, const double *qz,
                          double *vx, double *vy, double *vz, double dt,
                          double eps, double Sc, void *stream);

/* Relative L2 change, l2_norm (tse.py:273-281), NaN -> 1; result written to
 * d_out[0].  Replaces tse.py:273. */
int32_t tse_l2_norm(const double *New, const double *Old, int64_t n,
                    double *d_out, void *d_workspace, size_t workspace_bytes,
                    void *stream);

/* CFL limit of the driver (tse.py:1241-1249), reshape semantics included;
 * d_out[0] = dt_CFL.  Replaces tse.py:1241-1249. */
int32_t tse_dt_cfl(const TseGrid *grid, const double *qx, const double *qy,
                   const double *qz, const double *phi, double *d_out,
                   void *d_workspace, size_t workspace_bytes, void *stream);

/* Neumann limit explicit_C (tse.py:385-396) over nspec (<= 8) species
 * arrays; h_D is a HOST array of nspec device pointers; d_out[0] = dt_NeC.
 * Replaces tse.py:385. */
int32_t tse_explicit_C(const TseGrid *grid, const double *const *h_D,
                       int32_t nspec, const double *phi, double *d_out,
                       void *d_workspace, size_t workspace_bytes, void *stream);

/* Field statistics used by the driver (species skip test tse.py:1300-1301,
 * printout tse.py:1280-1285): d_out = {sum, max, min} in FP64, NaN
 * propagating for max/min like numpy. */
int32_t tse_field_stats(const double *x, int64_t n, double *d_out,
                        void *d_workspace, size_t workspace_bytes, void *stream);

/* Declared linear equation of state, the GPU form of the per-cell callback
 * run by run_fluid_properties (tse.py:179-199):
 *   rho_f = rho0 + a[0]*C[s[0]] + ... + a[m-1]*C[s[m-1]] - tcoef*(T - T0)
 * evaluated left to right (m <= 8 terms).  h_C is a HOST array of species
 * device pointers indexed by h_sidx. */
int32_t tse_eos_linear(const TseGrid *grid, const double *const *h_C,
                       const int32_t *h_sidx, const double *h_coef, int32_t m,
                       const double *T, double rho0, double tcoef, double T0,
                       double *rho_f, void *stream);

/* Declared per-cell property forms, the GPU form of further callbacks run by
 * run_fluid_properties (tse.py:179-199), e.g. the temperature polynomials of
 * course/04-groundwater_heat_tracer_eos/config.py:118-124, 197-219:
 *   TSE_EOS_CONSTANT  out = coef[0]
 *   TSE_EOS_POLY4_T   out = coef[4] + coef[3]*T + coef[2]*T**2 + coef[1]*T**3
 *                           + coef[0]*T**4   (numpy.polyfit order), left to
 *                     right, with T**3 = T*(T*T) and T**4 = (T*T)*(T*T) as
 *                     numba computes literal integer powers.
 * guard (device field or NULL): cells where guard == guard_value keep their
 * value (the callback's `if C[s] != v:`).  T may be NULL for a constant. */
#define TSE_EOS_CONSTANT 1
#define TSE_EOS_POLY4_T 2
typedef struct TseEosForm {
  int32_t kind;
  int32_t reserved;
  double guard_value;
  double coef[5];
} TseEosForm;
int32_t tse_eos_form(const TseGrid *grid, const TseEosForm *form, const double *T,
                     const double *guard, double *out, void *stream);

/* Peclet maxima peclet_C / peclet_T (tse.py:331-383), printed diagnostics:
 * d_out[0..2] = max Pe_x, Pe_y, Pe_z over non-boundary cells (NaN
 * propagating; cells on the boundary count as 0 as the zero-initialised
 * arrays of the reference do).  h_Dx/h_Dy/h_Dz are HOST arrays of nspec
 * (<= 8) device pointers. */
int32_t tse_peclet_C(const TseGrid *grid, const double *qx, const double *qy,
                     const double *qz, const double *const *h_Dx,
                     const double *const *h_Dy, const double *const *h_Dz,
                     int32_t nspec, const double *BC, double *d_out,
                     void *d_workspace, size_t workspace_bytes, void *stream);
int32_t tse_peclet_T(const TseGrid *grid, const double *qx, const double *qy,
                     const double *qz, const double *rho_f, const double *cp_f,
                     const double *phi, const double *l_r, const double *l_f,
                     const double *BT, double *d_out, void *d_workspace,
                     size_t workspace_bytes, void *stream);

/* Mass-balance totals in FP64 (no counterpart kernel in the reference, whose
 * mass_balance is a user callback, tse.py:1460-1463): d_out receives, with
 * V = dx dy dz per cell,
 *   [0]            water   sum phi rho_f V
 *   [1..ns]        species sum RC phi C_s V
 *   [ns+1]         heat    sum (phi rho_f cp_f + (1-phi) rho_r cp_r) T V
 *   [ns+2]         source rate sum WP V
 *   [ns+3..2ns+2]  source rates sum WC_s V
 *   [2ns+3]        source rate sum WT V
 * h_C / h_WC are HOST arrays of nspec (<= 8) device pointers; workspace
 * TSE_WS_REDUCE. */
int32_t tse_mass_totals(const TseGrid *grid, const double *phi,
                        const double *rho_f, const double *RC,
                        const double *const *h_C, const double *const *h_WC,
                        int32_t nspec, const double *T, const double *cp_f,
                        const double *rho_r, const double *cp_r,
                        const double *WP, const double *WT, double *d_out,
                        void *d_workspace, size_t workspace_bytes, void *stream);

/* Self-test of the bounded waits (no counterpart in the reference).  Every
 * persistent kernel here waits on other blocks (grid barriers) or on its own
 * bulk copies (mbarriers), and each of those waits gives up after a time
 * limit, raises an error flag and lets the kernel return with
 * TSE_STATUS_BARRIER_TIMEOUT.  This call runs each kind of wait -- the
 * generation grid barrier, the counter grid barrier, the mbarrier wait --
 * against a condition that never comes true, with a limit of timeout_s
 * seconds (at most 5), and writes to d_result[0..2] 1 for each wait that gave
 * up and raised its flag, 0 otherwise.  d_ws: at least 512 bytes of device
 * memory.  Takes about 3 * timeout_s; nothing faults or hangs. */
int32_t tse_selftest_bounded_waits(int32_t *d_result, double timeout_s, void *d_ws,
                                   size_t ws_bytes, void *stream);

/* Batched solves run so far by the fused form's device-driven loop and by its
 * host loop (TseDcOptions.host_loop; no counterpart in the reference). */
int32_t tse_batch_loop_stats(int64_t *graph_solves, int64_t *host_solves);

/* Library version string. */
const char *tse_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TSE_CUDA_H */
