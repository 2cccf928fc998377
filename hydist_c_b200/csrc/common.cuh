// common.cuh -- shared device-side types of the B200 Hydist time step.
//
// Layout in HBM: every mesh field is one FP64 (or int32) array of
// (N+3) x (M+3), row-major, idx = i*W + j with W = M+3 (the reference's
// layout, engine.h:56-68). Rows i are the x direction, columns j the y
// direction (contiguous). A column sweep (x, implicit in i) therefore maps
// one thread to one column and is coalesced across a warp; a row sweep
// (y, implicit in j) stages rows through shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hydist_capi.h"

namespace hyd {

constexpr int SEG = HYDIST_SEGMENT_LIMIT;

// Constant_Coeffs (engine.h:39-52), derived as Load_coeffs does, in the
// arithmetic type R of the step (double; float in the FP32 form).
template <class R>
struct CoefT {
  R dX, dY, dT, dXbp, dYbp, dX2, dY2, dTchia2dX, dTchia2dY, HaiChiadT;
  R NANGDAY, H_TINH, heso, mu_mn, kenhhepng, kenhhepd;
  R NDnen, Tod, Toe, hstoe, ghtoe, Mbochat;
  R ro, ros, dm, muy, d90, Dorong, Sx;
  R CORIOLIS_FORCE, g, Ks, Windx, Windy, Ufr, Dxr, wss;
  // reciprocals and products of constants, so that the kernels multiply
  // where the reference divides by a constant (one rounding of difference)
  R r_dX, r_dY, r_dX2, r_dY2, r_dXbp, r_dYbp, dT_dXbp, dT_dYbp, sqrt_g;
  R Mb_ros, r_Tod, r_Ufr2, Dxr_m03;  // Mbochat/ros, 1/Tod, 1/Ufr^2, Dxr^-0.3
  R qb_k;  // 0.053 sqrt((Sx-1) g) dm^1.5 of the bed-load flux

  template <class Q>
  static CoefT from(const CoefT<Q>& q) {
    CoefT c;
    const Q* src = reinterpret_cast<const Q*>(&q);
    R* dst = reinterpret_cast<R*>(&c);
    for (size_t k = 0; k < sizeof(CoefT<Q>) / sizeof(Q); ++k) dst[k] = (R)src[k];
    return c;
  }
};
using Coef = CoefT<double>;

// Device error flags recorded (or-ed) in State::err[0]: a line with more
// wet segments than the tables hold; a non-finite value committed to the
// state (NaN/Inf canary of the commits).
enum DevErr { DEV_OK = 0, DEV_SEG_OVERFLOW = 1, DEV_NONFINITE = 2 };

// Records a non-finite committed value (the store of the flag runs only
// when one is found).
template <class T>
__device__ __forceinline__ void canary(int* err, T a, T b, T c) {
  if (!(isfinite(a) && isfinite(b) && isfinite(c))) atomicOr(err, DEV_NONFINITE);
}

// Every device pointer of one scenario. Passed by value to kernels. The
// water level (z, t_z), the bed (h, htaiz, htaiz_bd, dH), the series and the
// clock are FP64 in every form; the other fields have the type R of the step
// (double in the plain form, float in the FP32 form).
template <class R>
struct StateT {
  int M, N, W, H;  // W = M+3, H = N+3
  int T;           // rows of the hourly series
  int bienQ[4];
  int ketdinh;
  int race_new;    // extraction at an open last end reads the new neighbour
  int refine;      // line solves refined once with an FP64 residual
  // boundary update: 0 the hourly series (Update_Boundary_Value); in the
  // narrow-channel mode 1 none (update_boundary_at_t, engine.cpp:24-30) or
  // 2 the standing wave of boundary_up/down/left/right
  int chan;
  // line ranges of the hydraulic sweeps: columns x_lo..x_hi (x sweep), rows
  // y_lo..N (y sweep); 3..M-1 / 3..N in the narrow-channel mode
  int x_lo, x_hi, y_lo;
  int reset_h;     // Reset_states_horizontal in the first half-step
  int bed_fb;      // the bed change feeds back into h, htaiz, Kx1, Ky1
  double src_start;  // the concentration sweeps' erosion source from this time
  const double *h0, *htaiz0;  // the initial bed (with bed_fb)
  // static fields
  const double *h, *hsnham, *htaiz, *htaiz_bd;
  const R *visco, *Fw, *Kx1, *Ky1, *Tsxw, *Tsyw;
  // state
  double *z, *tz, *dH;
  R *u, *v, *tu, *tv, *Hmoi, *Htdu, *Htdv, *FS, *tFS, *VTH, *Kx, *Ky, *Qbx, *Qby;
  int* khouot;
  // boundary
  R *ubt, *ubp, *vbt, *vbd;
  double *hi, *hmax;  // hmax[4]: up, down, left, right
  const double *bc[4], *CC[4];
  const int* btype;  // 4 x SEG
  // wet segments
  int *daui, *cuoii, *moci, *dauj, *cuoij, *mocj;
  // scratch
  R* tmp;        // smoothing buffer, (N+3)*(M+3)
  R *su, *sv;    // t_u / t_v after the smoothing of the current half-step
  int* err;      // [0]: DevErr
  R* lscratch;   // partitioned line solver: one slot per resident CTA
  // the rows of the next concentration sweep (A, B, C, D of every cell:
  // four arrays of (N+3)*(M+3), array k at pre + k*W*H)
  R* pre;
  int lslots;    // number of slots (CTAs of the persistent sweep grid)
  int* colflag;  // per column: holds a cell dried during the run
  int* rowflag;  // per row: the same (wetting along rows)
  int* segcnt;   // run-start / run-end counters of the segment scan
  double* clock; // [0]: simulated time, advanced on the device by k_tick
};
using State = StateT<double>;

// Many scenarios of one mesh size stepped by the same launches: the states
// and coefficients of the members in device arrays; a kernel launched for
// the batch takes member blockIdx.z (the line solvers: the member of the
// line group). n = 0: one scenario, passed by value.
template <class R>
struct Batch {
  const StateT<R>* S = nullptr;
  const CoefT<R>* c = nullptr;
  int n = 0;
};

// Bounds of the per-cell kernels with many operands (128-thread CTAs). A
// batch variant reads its member's StateT/CoefT from global memory, not the
// parameter bank, and ptxas holds the loaded pointers in registers (84 to 124
// of them in FP64); capped at 64, eight CTAs per SM: the 64-member ensemble
// of 1024x512 steps in 14.9 against 16.9 ms (FP64), 10.35 against 10.69
// (FP32), 12.28 against 12.63 (FP32 refined), their few spills in L1. The
// single-scenario kernels are separate entry points without the bound.
#define HYD_CELL_BOUNDS __launch_bounds__(128, 8)

// The state and coefficients a kernel works on: its by-value arguments, or
// with BATCH those of member blockIdx.z.
template <int BATCH, class R>
__device__ __forceinline__ StateT<R> member_state(const StateT<R>& S0, const Batch<R>& b) {
  if constexpr (BATCH != 0) return b.S[blockIdx.z];
  else return S0;
}
template <int BATCH, class R>
__device__ __forceinline__ CoefT<R> member_coef(const CoefT<R>& c0, const Batch<R>& b) {
  if constexpr (BATCH != 0) return b.c[blockIdx.z];
  else return c0;
}

// grid z of a launch: one slice per member of a batch
template <class R>
inline unsigned grid_z(const Batch<R>& b) { return b.n > 0 ? (unsigned)b.n : 1u; }

__host__ __device__ inline int cdiv(int a, int b) { return (a + b - 1) / b; }

// Phases of one full step, in launch order (engine.cpp:65-295).
enum Phase {
  PH_BOUNDARY_X = 0,  // Update_Boundary_Value, first half
  PH_SWEEP_X,         // x sweep: assembly + tridiagonal solve + extraction
  PH_EXPLICIT_V,      // smoothing of u, explicit v, margins, smoothing of v
  PH_COMMIT_X,        // H_moi, commit, total depths (and, before a concentration
                      // step, the speed and diffusivities)
  PH_SEDIMENT_X,      // concentration i-sweep, commit
  PH_BOUNDARY_Y,
  PH_SWEEP_Y,
  PH_EXPLICIT_U,
  PH_COMMIT_Y,        // + wetting/drying, segment tables
  PH_SEDIMENT_Y,
  PH_COUNT
};

// The line-solver launches of one step, timed one by one when traced.
enum SweepKernel {
  KS_SWEEP_X = 0,  // hydraulic x sweep
  KS_SWEEP_Y,      // hydraulic y sweep
  KS_FS_X,         // concentration x sweep
  KS_FS_Y,         // concentration y sweep
  KS_COUNT
};

// Launch bookkeeping: counts kernels and, when events are given, records
// an event at the end of each phase and around each line-solver launch (the
// tracing of hydist_step_traced / hydist_step_traced_sweeps).
struct Trace {
  cudaEvent_t* ev = nullptr;   // PH_COUNT + 1 events; ev[0] = step start
  cudaEvent_t* kev = nullptr;  // 2 * KS_COUNT events: begin, end of each sweep
  bool krec[KS_COUNT] = {};
  long long launches = 0;
  void mark(cudaStream_t st, int phase, int nkernels) {
    launches += nkernels;
    if (ev) cudaEventRecord(ev[phase + 1], st);
  }
  void kbegin(cudaStream_t st, int k) {
    if (kev) cudaEventRecord(kev[2 * k], st);
  }
  void kend(cudaStream_t st, int k) {
    if (kev) {
      cudaEventRecord(kev[2 * k + 1], st);
      krec[k] = true;
    }
  }
};

}  // namespace hyd
