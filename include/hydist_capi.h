/*
 * hydist_capi.h -- C ABI of the B200 (sm_100a) implementation of the Hydist_C
 * ADI time step (2D shallow-water hydraulics + suspended-sediment transport)
 * and of its batched tridiagonal solver.
 *
 * Plain C: pointers, sizes and status codes only. Every function returns an
 * int status (HYDIST_OK = 0, negative on error; hydist_last_error() gives the
 * message of the calling thread's last failure). No exception crosses this
 * boundary.
 *
 * Data conventions are the reference's (engine.h:16-89, loader.cpp:224-375):
 *   - mesh fields are FP64, row-major (N+3) x (M+3), idx = i*(M+3) + j;
 *     i in [2,N] is the x / u / dX direction ("rows"), j in [2,M] is the
 *     y / v / dY direction ("columns", contiguous in memory);
 *   - the wet/dry mask (khouot) is int32 of the same shape: 0 wet, 1 dried
 *     during the run, 2 dry at initialisation;
 *   - boundary series are flat [segment * total_time + hour];
 *   - sides are indexed up (j = M), down (j = 2), left (i = 2), right (i = N).
 *
 * Which reference interface each entry point replaces is cited beside it as
 * reference-file:line (paths relative to the Hydist_C source tree).
 */
#ifndef HYDIST_CAPI_H
#define HYDIST_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HYDIST_SEGMENT_LIMIT 20 /* wet segments per line, engine.h:12 */

/* ---- status codes ---------------------------------------------------- */
enum HydistStatus {
  HYDIST_OK = 0,
  HYDIST_ERR_ARG = -1,        /* bad argument (null pointer, size, enum)   */
  HYDIST_ERR_CUDA = -2,       /* a CUDA runtime call failed                */
  HYDIST_ERR_OOM = -3,        /* device allocation failed                  */
  HYDIST_ERR_SEGMENTS = -4,   /* a line has more than 20 wet segments      */
  HYDIST_ERR_STATE = -5,      /* call not valid in the handle's state      */
  HYDIST_ERR_BUDGET = -6,     /* serving: request exceeds the HBM budget   */
  HYDIST_ERR_TIMEOUT = -7,    /* a bounded device wait gave up             */
  HYDIST_ERR_NONFINITE = -8,  /* NaN/Inf detected in the state             */
  HYDIST_ERR_NODEVICE = -9    /* no CUDA device visible                    */
};

/* ---- fields exchangeable with the host ------------------------------- */
enum HydistField {
  HYDIST_FIELD_U = 0,      /* u  (Argument_Pointers::u)                    */
  HYDIST_FIELD_V = 1,      /* v                                            */
  HYDIST_FIELD_Z = 2,      /* z  water level                               */
  HYDIST_FIELD_FS = 3,     /* suspended concentration (volumetric)         */
  HYDIST_FIELD_TFS = 4,    /* concentration sweep buffer (tFS)             */
  HYDIST_FIELD_H_MOI = 5,  /* total depth at z points                      */
  HYDIST_FIELD_KHOUOT = 6, /* int32 wet/dry mask                           */
  HYDIST_FIELD_DH = 7,     /* accumulated bed change                       */
  HYDIST_FIELD_HTDU = 8,   /* total depth at u points                      */
  HYDIST_FIELD_HTDV = 9,   /* total depth at v points                      */
  HYDIST_FIELD_TU = 10,    /* t_u (provisional u)                          */
  HYDIST_FIELD_TV = 11,    /* t_v                                          */
  HYDIST_FIELD_TZ = 12,    /* t_z                                          */
  HYDIST_FIELD_KX1 = 13,   /* friction coefficient at u points             */
  HYDIST_FIELD_KY1 = 14,   /* friction coefficient at v points             */
  HYDIST_FIELD_VTH = 15,   /* speed at cell centre                         */
  HYDIST_FIELD_KX = 16,    /* sediment diffusivity, x                      */
  HYDIST_FIELD_KY = 17,    /* sediment diffusivity, y                      */
  HYDIST_FIELD_H = 18,     /* bed depth at nodes (bandodosau)              */
  HYDIST_FIELD_HTAIZ = 19, /* bed depth at z points                        */
  HYDIST_FIELD_QBX = 20,   /* bed-load flux, x                             */
  HYDIST_FIELD_QBY = 21,   /* bed-load flux, y                             */
  HYDIST_FIELD_COUNT = 22
};

/* Precision of the time step. */
enum HydistPrecision {
  HYDIST_FP64 = 0,       /* plain FP64 form: reproduces the reference       */
  HYDIST_FP32_REFINE = 1, /* FP32 fields, assembly and solves, each line
                             solve refined once with a residual computed in
                             FP64; FP64 water level, bed, series and mass
                             accumulation                                  */
  HYDIST_FP32 = 2         /* the same without the refinement pass          */
  /* hydist_create_external takes HYDIST_FP64 only */
};

/* Physical and numerical constants: the inputs of Load_coeffs
 * (loader.cpp:4-87, struct Constant_Coeffs engine.h:39-52). The derived
 * constants (dXbp, dTchia2dX, Ufr, Dxr, ...) are computed from these exactly
 * as Load_coeffs does. hydist_params_default() fills the reference values. */
typedef struct HydistParams {
  double dX, dY, dT;
  double NANGDAY;   /* bed-raise offset                      loader.cpp:22 */
  double H_TINH;    /* dry threshold (m)                     loader.cpp:23 */
  double heso;      /* smoothing weight                      loader.cpp:33 */
  double mu_mn;     /* Manning exponent parameter            loader.cpp:34 */
  double NDnen;     /* background concentration              loader.cpp:36 */
  double Tod, Toe, hstoe, ghtoe, Mbochat; /*                 loader.cpp:46-50 */
  double ro, ros;                         /*                 loader.cpp:53-54 */
  double dm, d90, muy, Dorong, Sx;        /*                 loader.cpp:57-66 */
  double CORIOLIS_FORCE, g;               /*                 loader.cpp:75-76 */
  double Wind, huonggio;                  /*                 loader.cpp:26-27 */
  double wss; /* settling velocity; < 0 derives it as loader.cpp:86      */
  double Ks;  /* roughness height; < 0 derives 2.5*dm as loader.cpp:79    */
} HydistParams;

/* Run options: the fields of struct Options (engine.h:16-37) that the time
 * step reads. */
typedef struct HydistOptions {
  double t_start;          /* simulated start time (s)         main.cpp:100 */
  double sediment_start;   /* -b: sediment sweeps from this t  main.cpp:82  */
  double bed_change_start; /* -B: erosion source and bed change from this t */
  int32_t ketdinh;         /* cohesive sediment (main.cpp:53 sets 1)        */
  int32_t bed_change;      /* 1: accumulate the bed change dH once per step
                              from bed_change_start (Calculate_Qb/BedLoad,
                              sediment_transport.cpp:352-537, which the
                              reference never launches)                     */
  int32_t precision;       /* enum HydistPrecision                          */
  /* narrow-channel mode (Options::kenhhepd / kenhhepng, engine.h:19-33;
     main.cpp flags -kd / -kn). With exactly one of the two set (the
     reference's `channel`), the boundary series are not applied
     (update_boundary_at_t does nothing, engine.cpp:24-30), and the x sweep
     takes columns 3..M-1 (kenhhepd, engine.cpp:77-80) or the y sweep rows
     3..N (kenhhepng, :190-193) instead of 2..M / 2..N. */
  int32_t kenhhepd, kenhhepng;
  /* 1: in channel mode, impose the standing-wave water levels of
     boundary_up / boundary_down / boundary_left / boundary_right
     (support_funcs.cpp:366-478) at every half-step, as the calls the
     reference keeps commented out at engine.cpp:25-28 would */
  int32_t channel_wave;
  /* 1: wetting and drying along rows as well: Reset_states_horizontal
     (support_funcs.cpp:88-138, which the reference never launches) after
     update_h_moi in the first half-step, the place Reset_states_vertical
     takes in the second (engine.cpp:238-240) */
  int32_t reset_horizontal;
  /* 1 (with bed_change): the accumulated bed change feeds back into the
     bed: htaiz = htaiz0 + dH at z points, the node depths h and the
     friction coefficients Kx1, Ky1 (support_funcs.cpp:21-69) follow
     once per step */
  int32_t bed_feedback;
  int32_t reserved;
} HydistOptions;

/* One scenario's inputs, host pointers, in the reference's text-input
 * meaning (loader.cpp:120-168). Series hold at least total_time entries for
 * segment 0 (the only segment the reference's boundary update reads,
 * support_funcs.cpp:614-618). All pointers are read during the call only. */
typedef struct HydistScenario {
  int32_t M, N;               /* interior extents; arrays are (N+3)x(M+3)     */
  int32_t total_time;         /* rows of the hourly series (loader.cpp:165)   */
  int32_t n_boundary_type;    /* entries in boundary_type (80 = 4 sides x 20) */
  const double* h;            /* bandodosau: bed depth at nodes               */
  const double* hsnham;       /* Manning roughness                            */
  const double* visco;        /* hsnhotroiA: eddy viscosity (VISCOIDX)        */
  const double* Fw;           /* Fw_map                                       */
  const double* bc_up;        /* hourly Z or Q series per side                */
  const double* bc_down;
  const double* bc_left;
  const double* bc_right;
  const double* CC_up;        /* hourly FS boundary series per side           */
  const double* CC_down;
  const double* CC_left;
  const double* CC_right;
  const int32_t* boundary_type; /* side-major, 20 per side; 2 = discharge     */
  int32_t bienQ[4];           /* discharge flag per side (up,down,left,right)
                                 as loader.cpp:157-164 derives it            */
  const double* FS0;          /* optional initial concentration, or NULL      */
  const double* z0;           /* optional initial water level (z and t_z
                                 before the set-up kernels; the reference
                                 starts from the zeroed allocation,
                                 loader.cpp:269-271), or NULL               */
} HydistScenario;

typedef struct HydistHandle HydistHandle;

/* Reference constants of Load_coeffs (loader.cpp:4-87). */
void hydist_params_default(HydistParams* p);
/* Options as main.cpp:49-53 defaults them (t_start 0, ketdinh 1, FP64). */
void hydist_options_default(HydistOptions* o);
/* bienQ[k] = (boundary_type[k] == 2) for k < 4, as loader.cpp:157-164. */
void hydist_bienq_from_boundary_type(const int32_t* boundary_type, int32_t n,
                                     int32_t bienQ[4]);

const char* hydist_last_error(void);
const char* hydist_version(void);

/* ---- one scenario on the device --------------------------------------
 * hydist_create replaces the set-up sequence of main.cpp:138-304
 * (attribute_arrays_memory_alloc loader.cpp:224-330, supporting_arrays_alloc
 * loader.cpp:333-375, Load_coeffs, Onetime_init support_funcs.cpp:21-69,
 * Find_Calculation_limits_* :238-343, Htuongdoi :346-362, preprocess_data
 * :482-601). All device state is allocated here and freed by hydist_destroy.
 * device < 0 uses the current device. */
int hydist_create(const HydistScenario* sc, const HydistParams* p,
                  const HydistOptions* o, int device, HydistHandle** out);
int hydist_destroy(HydistHandle* h);

/* Device arrays of one scenario owned by the caller, in the reference's
 * layout: the arrays of Argument_Pointers (engine.h:56-72) after the
 * reference's set-up (main.cpp:260-309: Onetime_init, the segment scans,
 * Htuongdoi). bienQ holds the four discharge flags as values. */
typedef struct HydistExternal {
  int32_t M, N, total_time;
  int32_t bienQ[4];
  /* read only */
  const double *h, *hsnham, *visco, *Fw, *htaiz, *htaiz_bd, *Kx1, *Ky1, *Tsxw, *Tsyw;
  const double *bc_up, *bc_down, *bc_left, *bc_right;
  const double *CC_up, *CC_down, *CC_left, *CC_right;
  const int32_t* boundary_type; /* 4 sides x 20 segments */
  /* state, read and written in place */
  double *u, *v, *z, *t_u, *t_v, *t_z, *H_moi, *Htdu, *Htdv;
  double *FS, *tFS, *VTH, *Kx, *Ky, *dH, *Qbx, *Qby;
  int32_t *khouot, *daui, *cuoii, *moci, *dauj, *cuoij, *mocj;
  double *ubt, *ubp, *vbt, *vbd;
} HydistExternal;

/* A handle over caller-owned device state (the reference's ownership:
 * loader.cpp:224-375 allocates, the time loop works in place). Nothing of
 * the caller's is copied or freed; the library allocates only its own
 * scratch (smoothing buffers, line-solver scratch, the boundary discharge
 * weights of preprocess_data, which it recomputes from h and htaiz_bd).
 * The arrays must stay valid until hydist_destroy. */
int hydist_create_external(const HydistExternal* ext, const HydistParams* p,
                           const HydistOptions* o, int device,
                           HydistHandle** out);

/* Advance nsteps full ADI steps (two half-steps each): the body of the time
 * loop of Hydraulic_Calculation (engine.cpp:65-295). Stream-ordered on the
 * handle's stream; returns once the work is enqueued. */
int hydist_step(HydistHandle* h, int32_t nsteps);

/* One half of a step: half 0 = t += dT/2, the x sweep (UZ), explicit v,
 * commit and the concentration i-sweep (engine.cpp:65-171); half 1 = the y
 * sweep (VZ), explicit u, wetting/drying, commit and the concentration
 * j-sweep (:175-288). Halves alternate 0, 1, 0, ...; a full-step call while
 * half 1 is pending returns HYDIST_ERR_STATE. */
int hydist_half_step(HydistHandle* h, int32_t half);

/* The boundary update at time t alone: update_boundary_at_t
 * (engine.cpp:22-36) / Update_Boundary_Value (support_funcs.cpp:603-728).
 * The handle's time is unchanged. */
int hydist_update_boundary(HydistHandle* h, double t);
/* Block until the handle's stream is idle (synch_and_check, engine.cpp:13). */
int hydist_sync(HydistHandle* h);
/* Simulated time of the state (seconds); set_time supports resuming a
 * checkpoint (the reference's -T start time, main.cpp:100-102). */
int hydist_get_time(HydistHandle* h, double* t);
int hydist_set_time(HydistHandle* h, double t);
/* Copy one field (HydistField) to/from host memory of (N+3)*(M+3) elements
 * (int32 for KHOUOT, double otherwise). Synchronous. Uploading KHOUOT
 * recomputes the wet-segment tables from it. */
int hydist_download(HydistHandle* h, int32_t field, void* host);
int hydist_upload(HydistHandle* h, int32_t field, const void* host);
/* Water volume sum over wet cells of (htaiz + z) * dX * dY, accumulated in
 * FP64 on the device (mass-conservation check). */
int hydist_mass(HydistHandle* h, double* volume);
/* Run nsteps with each step captured once into a CUDA graph and replayed.
 * Same results as hydist_step. */
int hydist_step_graph(HydistHandle* h, int32_t nsteps);
/* The CUDA stream the handle enqueues on (a cudaStream_t). */
void* hydist_stream(HydistHandle* h);

/* ---- checkpoint / resume ----------------------------------------------
 * The reference's resume is a stub (main.cpp:283-284). A checkpoint holds
 * the time and every field that carries from one step to the next, in a
 * binary file (header + FP64 fields + the int32 mask). Load restores them
 * into a handle created for the same scenario (same mesh and inputs) and
 * rescans the segment tables from the mask; stepping on is bit-identical to
 * not having stopped. Both are synchronous and allowed between full steps. */
int hydist_checkpoint_save(HydistHandle* h, const char* path);
int hydist_checkpoint_load(HydistHandle* h, const char* path);

/* ---- ensembles (the reference has none) ---------------------------------
 * Many scenarios on one device stepped together, one CUDA graph replay per
 * step. Members of one mesh size, form and launch-shaping options
 * (narrow-channel ranges, horizontal wetting, bed feedback) are batched:
 * each kernel of the step is one launch over all members (the per-cell
 * kernels take member blockIdx.z, the persistent line solvers walk the
 * line groups of every member), whenever the members are in the same
 * sediment phase. Otherwise one step of every member is captured with the
 * members' launches on their own streams, forked from the ensemble's stream
 * and joined back, so that they overlap on the device. A graph is captured
 * per pattern of the members' sediment phases. Members keep their own
 * handles (download, mass, ...); their own stream work before and after an
 * ensemble step is ordered with it. The ensemble does not own the members.
 * Results are those of stepping each member alone: bit for bit through the
 * members' own launches; to rounding when batched (the batched kernels are
 * separately compiled variants: about 1e-13 of a field's magnitude after
 * 30 steps in FP64). */
typedef struct HydistEnsemble HydistEnsemble;
int hydist_ensemble_create(HydistHandle* const* members, int32_t n,
                           HydistEnsemble** out);
int hydist_ensemble_step(HydistEnsemble* e, int32_t nsteps);
int hydist_ensemble_sync(HydistEnsemble* e);
/* The stream the ensemble's graphs are launched on (a cudaStream_t). */
void* hydist_ensemble_stream(HydistEnsemble* e);
/* enable = 0: step the members by their own launches even where they could
 * be batched; 1: batch them again (HYDIST_ERR_ARG if they differ in mesh
 * size, form or launch options). Batching is on after create where allowed. */
int hydist_ensemble_batched(HydistEnsemble* e, int32_t enable);
int hydist_ensemble_destroy(HydistEnsemble* e);

/* ---- serving (the reference has none) ------------------------------------
 * Continuous batching of scenario solves on one device. A request is a
 * scenario (host inputs copied at submit; the pointers are not kept) and a
 * horizon in steps. hydist_server_round: admits queued requests in arrival
 * order while their device footprint fits the budget; advances every active
 * request by up to steps_per_round steps, the requests of one mesh size and
 * form that advance alike stepped as an ensemble (their kernels launched
 * together for all of them, see hydist_ensemble_*), each group and each lone
 * request on its own stream (their kernels overlap on the device); waits;
 * retires those at their horizon and returns their ids. A retired request keeps its device state (and its share
 * of the budget) until hydist_server_release; hydist_server_handle gives its
 * handle for hydist_download / hydist_mass. Each request is computed by its
 * own handle: its result is the same alone and in the mix, bit for bit where
 * it steps alone, to rounding where its group steps as a batch (as for
 * ensembles). */
typedef struct HydistServer HydistServer;
enum HydistRequestState { HYDIST_RQ_QUEUED = 0, HYDIST_RQ_ACTIVE = 1, HYDIST_RQ_DONE = 2 };
/* Device bytes hydist_create allocates for an M x N scenario (upper bound). */
int64_t hydist_scenario_bytes(int32_t M, int32_t N);
int hydist_server_create(int device, uint64_t budget_bytes, int32_t steps_per_round,
                         HydistServer** out);
int hydist_server_destroy(HydistServer* s);
/* HYDIST_ERR_BUDGET if the scenario alone exceeds the budget. */
int hydist_server_submit(HydistServer* s, const HydistScenario* sc,
                         const HydistParams* p, const HydistOptions* o,
                         int32_t nsteps, int64_t* id);
int hydist_server_round(HydistServer* s, int64_t* done, int32_t cap, int32_t* ndone);
int hydist_server_status(HydistServer* s, int64_t id, int32_t* state, int32_t* steps_done);
int hydist_server_counts(HydistServer* s, int32_t* queued, int32_t* active,
                         uint64_t* held_bytes);
HydistHandle* hydist_server_handle(HydistServer* s, int64_t id);
int hydist_server_release(HydistServer* s, int64_t id);

/* Tracing (the reference has none): run one full step with a CUDA event at
 * the end of each phase and return the device time of each phase in ms, in
 * the order boundary-x, sweep-x, explicit-v, commit-x, sediment-x,
 * boundary-y, sweep-y, explicit-u, commit-y, sediment-y (HYDIST_PHASES
 * entries). Synchronous. */
#define HYDIST_PHASES 10
int hydist_step_traced(HydistHandle* h, float* phase_ms);
/* The same, also timing each line-solver launch of the step on its own:
 * sweep_ms[HYDIST_SWEEPS] = hydraulic x sweep, hydraulic y sweep,
 * concentration x sweep, concentration y sweep (0 for a sweep the step did
 * not run). */
#define HYDIST_SWEEPS 4
int hydist_step_traced_sweeps(HydistHandle* h, float* phase_ms, float* sweep_ms);
/* Host time of the handle's hydist_create by part, in ms (the reference
 * has no counterpart): ms[0] device allocation and zeroing (the arrays come
 * from a per-device memory pool that keeps what destroyed handles release),
 * ms[1] copies of the host inputs, ms[2] set-up kernels (Onetime_init,
 * segment tables, Htuongdoi, preprocess_data), ms[3] the whole call. */
int hydist_create_phases(const HydistHandle* h, double* ms);
/* Number of kernels the handle has enqueued since creation (set-up
 * excluded). */
int hydist_kernel_launches(HydistHandle* h, int64_t* count);

/* ---- batched tridiagonal solver --------------------------------------
 * Replaces tridiag() + tridiagSolver (UVZSolver_multithread.cpp:19-43,
 * 78-109) and gtsv_spike_partial_diag_pivot_v1 (gtsv.cpp:88-193) with one
 * batched, host-callable entry point. System s occupies rows
 * [offsets[s], offsets[s] + lengths[s]) of the packed arrays; dl[first row]
 * and du[last row] of each system are ignored. Arrays are device pointers.
 * dtype: 0 = FP64, 1 = FP32. algo (enum HydistGtsvAlgo):
 *   AUTO       per length band, the solver hydist_gtsv_autotune chose on
 *              this device (before any tuning: WARP up to 512 rows, then
 *              PARTITION_512 or PARTITION where the system fits a CTA's
 *              shared memory, THOMAS beyond);
 *   THOMAS     one thread per system, in place in global memory;
 *   PARTITION  one 256-thread CTA per system staged in shared memory:
 *              chunked Thomas with the chunk separators' reduced system
 *              solved by parallel cyclic reduction (SPIKE-style partition,
 *              no pivoting);
 *   WARP       one warp per system staged in shared memory, partition with
 *              a shuffle PCR of 32 separators (systems up to 512 rows);
 *   PARTITION_512  PARTITION with 512-thread tiles (more warps per system,
 *              less shared memory left for long systems).
 * A solver that cannot take a band's lengths passes it on (WARP ->
 * PARTITION_512 -> PARTITION -> THOMAS; PARTITION_128 -> PARTITION).
 * PARTITION_128, PARTITION and PARTITION_512 are the same CTA partition
 * solver on 128, 256 or 512 threads per system: fewer threads give each
 * thread a longer chunk and the separators a shorter reduction. Systems of length 0 are skipped.
 *   PIVOT      one thread per system, Gaussian elimination with diagonal
 *              pivoting (1x1 or 2x2 pivots by the Bunch-Kaufman criterion,
 *              kappa = (sqrt(5)-1)/2: the pivoting of the reference's SPIKE
 *              tile solver, spike_kernel.hxx:119-376), for systems that are
 *              not diagonally dominant; never chosen by AUTO.
 * The other solvers do not pivot: they expect diagonally dominant systems,
 * as the ADI sweeps' are.
 * stream is a cudaStream_t (NULL = default stream). The bands' solves run
 * side by side on the library's own streams, forked from `stream` and joined
 * back into it, so work queued on `stream` after the call waits for all of
 * them. Scratch is allocated by the library on first use and grown as
 * needed. The call synchronises the
 * stream once to read the band sizes and the packed extent, and, when a
 * shared-memory CTA solver (PARTITION*) ran, once more at the end: every
 * wait of those solvers for a system's rows is bounded, and a CTA that gave
 * up leaves its remaining systems unsolved, which this call (not a later
 * one) reports as HYDIST_ERR_TIMEOUT. A batch with a negative offset is
 * refused with HYDIST_ERR_ARG. */
enum HydistGtsvAlgo {
  HYDIST_GTSV_AUTO = 0,
  HYDIST_GTSV_THOMAS = 1,
  HYDIST_GTSV_PARTITION = 2,
  HYDIST_GTSV_WARP = 3,
  HYDIST_GTSV_PARTITION_512 = 4,
  HYDIST_GTSV_PARTITION_128 = 5,
  HYDIST_GTSV_PIVOT = 6
};
int hydist_gtsv_batched(const void* dl, const void* d, const void* du,
                        const void* b, void* x, const int32_t* offsets,
                        const int32_t* lengths, int32_t nsys, int32_t dtype,
                        int32_t algo, void* stream);

/* The same solve for FP64 systems computed in FP32 with one refinement
 * whose residual is computed in FP64 (the refine option of the batched
 * solve; the reference has no counterpart): the systems are rounded to
 * FP32 and solved by `algo`'s FP32 solvers, r = b - A x is formed in FP64
 * from the FP64 arrays, the correction A d = r is solved in FP32 by the same
 * solvers and x + d is returned in FP64. Arrays as for
 * hydist_gtsv_batched with dtype 0; the library's scratch holds the FP32
 * copies (20 bytes per row). */
int hydist_gtsv_batched_refine(const double* dl, const double* d, const double* du,
                               const double* b, double* x, const int32_t* offsets,
                               const int32_t* lengths, int32_t nsys, int32_t algo,
                               void* stream);

/* Length bands of the batched solver: band b holds the systems with
 * hi[b-1] < length <= hi[b] (hi[-1] = 0), HYDIST_GTSV_BANDS entries. */
#define HYDIST_GTSV_BANDS 7
int hydist_gtsv_band_bounds(int32_t* hi);

/* Autotuner (the reference has none): for each length band, times every
 * solver that can take the band's lengths on a synthetic diagonally
 * dominant batch of that band (about 4M rows) on this device and keeps the
 * fastest for algo = AUTO. Allocates temporary device memory and
 * synchronises the stream. algo_per_band (may be NULL) receives the choice
 * per band. */
int hydist_gtsv_autotune(int32_t dtype, void* stream, int32_t* algo_per_band);

/* Allocation-free batched Thomas solve (no counterpart in the reference,
 * whose gtsv allocates per call). Same arrays and results as
 * hydist_gtsv_batched with algo = 1, for callers that must not allocate
 * device memory while they run. The forward-sweep scratch is a fixed array
 * of HYDIST_GTSV_NOALLOC_MAX_ROWS rows inside the library (8 MiB per device,
 * reserved when the library is loaded on the device); nothing is allocated
 * by any call.
 *   rows   packed rows of the arrays: every system must lie in [0, rows);
 *          a system outside is left unsolved. rows above the limit return
 *          HYDIST_ERR_BUDGET without launching anything.
 * The first call on each device (with that device current) looks up the
 * scratch address; make that call before capturing a stream. A call that
 * finds the device's context changed since (cudaDeviceReset) looks the
 * address up again, as a first call does. Nothing needs
 * zeroing beforehand. The scratch is shared by all calls on a device, so
 * calls that overlap in time on one device (two streams or host threads)
 * race and must be serialised by the caller. */
#define HYDIST_GTSV_NOALLOC_MAX_ROWS (1 << 20)
int hydist_gtsv_batched_noalloc(const void* dl, const void* d, const void* du,
                                const void* b, void* x, const int32_t* offsets,
                                const int32_t* lengths, int32_t nsys,
                                int32_t rows, int32_t dtype, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HYDIST_CAPI_H */
