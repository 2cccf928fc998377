// hydro.cu -- hydraulic ADI half-steps and the wet/dry bookkeeping on the GPU.
//
// Kernels (reference kernel each one replaces in brackets):
//   k_onetime_init      [Onetime_init, support_funcs.cpp:21-69]
//   k_interp_fs_rows    [Interpolate_FS_ng, support_funcs.cpp:191-213]
//   k_interp_fs_col     [Interpolate_FS_d, support_funcs.cpp:215-237]
//   k_runs_flags/sort   [Find_Calculation_limits_Horizontal/Vertical, :238-343]
//   k_htuongdoi         [Htuongdoi, :346-362] (set-up; per step in the commits)
//   k_preprocess_sides  [preprocess_data, :482-601]
//   k_boundary          [Update_Boundary_Value/Boundary_value/FS_boundary, :603-728;
//                        it also advances the device clock]
//   the line sweeps     [UZSolver_*/VZSolver_* + tridiagSolver,
//                        UVZSolver_multithread.cpp:19-139, 142-603, 798-933]:
//                        sweep.cu on the partitioned solver of linesolve.cuh
//   k_smooth_full       [Normalize/_normalize/update_buffer, :761-808]
//   k_solve_v/k_solve_u [solveV/vSolver, solveU/uSolver, :607-795, 938-978]
//   k_margin_v/k_margin_u [update_margin_elem_V/U, :980-1060]
//   k_commit_a          [update_h_moi + update_uvz + Htuongdoi, :71-86, 732-759, 346-362;
//                        before a concentration step also Find_VTH + hesoK,
//                        sediment_transport.cpp:575-602, 539-573]
//   k_smooth_full (with H_moi), k_wetting, k_commit_b, k_runs_flags (drying)
//                       [update_h_moi + Reset_states_vertical + update_uvz +
//                        Htuongdoi, support_funcs.cpp:71-86, 142-188, 732-759;
//                        Find_VTH + hesoK as in k_commit_a]
//
// Formulas keep the reference's structure; nvcc may fuse a multiply and an
// add into one FMA, which the CPU oracle does not, so results agree to
// rounding, not bit for bit.
#include <cstdio>

#include "assembly.cuh"
#include "common.cuh"
#include "explicit.cuh"
#include "hydro.cuh"
#include "sediment_cell.cuh"

namespace hyd {

// ----------------------------------------------------------------- init
template <class R>
__global__ void k_onetime_init(StateT<R> S, CoefT<R> c) {
  const int W = S.W, H = S.H, N = S.N, M = S.M;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (i >= H || j >= W) return;
  const int p = i * W + j;
  // borders and cells beyond the wet test are dry (2); row 0 / column 0
  int k = 2;
  double hm = 0.0;
  bool set_h = false;
  if (i >= 1 && j >= 1 && i <= N + 1 && j <= M + 1) {
    if ((S.h[(i - 1) * W + j - 1] + S.h[(i - 1) * W + j] + S.h[i * W + j - 1] + S.h[p]) * 0.25 >
        c.NANGDAY) {
      k = 0;
      set_h = true;
    }
  }
  S.khouot[p] = k;
  if (set_h) S.Hmoi[p] = hm;
  if (i >= 1 && j >= 1 && i <= N && j <= M) {
    double* htaiz = const_cast<double*>(S.htaiz);
    double* htaiz_bd = const_cast<double*>(S.htaiz_bd);
    R* Kx1 = const_cast<R*>(S.Kx1);
    R* Ky1 = const_cast<R*>(S.Ky1);
    htaiz[p] = (S.h[(i - 1) * W + j - 1] + S.h[(i - 1) * W + j] + S.h[i * W + j - 1] + S.h[p]) * 0.25;
    htaiz_bd[p] = htaiz[p];
    if (S.h[i * W + j - 1] + S.h[p] != 0)
      Kx1[p] = c.g * pow((S.h[i * W + j - 1] + S.h[p]) * 0.5, -2 * c.mu_mn) *
               pow((S.hsnham[i * W + j - 1] + S.hsnham[p]) * 0.5, 2.0);
    if (S.h[(i - 1) * W + j] + S.h[p] != 0)
      Ky1[p] = c.g * pow((S.h[(i - 1) * W + j] + S.h[p]) * 0.5, -2 * c.mu_mn) *
               pow((S.hsnham[(i - 1) * W + j] + S.hsnham[p]) * 0.5, 2.0);
  }
}

// ------------------------------------------------------- segment tables
template <class R, int BATCH = 0>
__global__ void k_interp_fs_rows(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  // Interpolate_FS_ng at row N (offset N-1, sign -1) and row 2 (offset 2, +1)
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int which = blockIdx.y;
  if (j >= S.M) return;
  const int W = S.W;
  const int loc = which == 0 ? S.N : 2;
  const int offset = which == 0 ? S.N - 1 : 2;
  const int sign = which == 0 ? -1 : 1;
  if (S.tu[loc * W + j] > 0) {
    const double deltaX = (S.u[loc * W + j] + S.tu[loc * W + j]) * 0.25 * c.dT;
    const double fi = offset + sign * (deltaX / c.dX);
    // a source row outside the mesh (reachable only once the state is no
    // longer finite) is skipped, never read
    if (!(fi > -1.0 && fi < (double)(S.H - 1))) return;
    const int i = (int)fi;
    const int i_deltaX = __double2int_rn(deltaX);
    const int i_dX = __double2int_rn(c.dX);
    S.FS[loc * W + j] = S.FS[i * W + j] +
                        sign * (S.FS[(i + 1) * W + j] - S.FS[i * W + j]) * (deltaX / c.dX - i_deltaX / i_dX);
  }
}

template <class R, int BATCH = 0>
__global__ void k_interp_fs_col(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  // Interpolate_FS_d at column M (offset M-1, sign -1); rows 1..M-1 as the
  // reference loops them (support_funcs.cpp:227)
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i >= S.M || i >= S.H) return;
  const int W = S.W, loc = S.M, offset = S.M - 1, sign = -1;
  if (S.tv[i * W + loc] > 0) {
    const double deltaY = (S.v[i * W + loc] + S.tv[i * W + loc]) * 0.25 * c.dT;
    const double fj = offset + sign * (deltaY / c.dY);
    if (!(fj > -1.0 && fj < (double)(W - 1))) return;
    const int j = (int)fj;
    const int j_deltaY = __double2int_rn(deltaY);
    const int j_dY = __double2int_rn(c.dY);
    S.FS[i * W + loc] = S.FS[i * W + j + 1] +
                        (S.FS[i * W + j + 1] - S.FS[i * W + j]) * (deltaY / c.dY - j_deltaY / j_dY);
  }
}

// The wet-segment tables of Find_Calculation_limits_* (support_funcs.cpp:
// 238-343) in parallel form. A cell p of a line (positions 2..lim) is
// the start of a recorded run when it is wet, p == 2 or p-1 is dry, and
// p <= lim-2; it is the end of a recorded run when it is wet, p == lim or
// p+1 is dry, and the run it ends starts at or before lim-2 (for p = lim-1
// that needs lim-2 wet, for p = lim both lim-2 and lim-1 wet). Starts and
// ends claim slots with atomics; k_runs_sort orders each line's slots.
// seg_cnt: [0..H) row starts, [H..2H) row ends, [2H..2H+W) column starts,
// [2H+W..2H+2W) column ends.
__device__ __forceinline__ void run_flags(bool wm1, bool w, bool wp1, bool wm2_lim, int p,
                                          int lim, bool& start, bool& end) {
  start = w && (p == 2 || !wm1) && p <= lim - 2;
  bool ok = true;
  if (p == lim - 1) ok = wm1;        // wm1 = wet(lim-2)
  else if (p == lim) ok = wm1 && wm2_lim;  // wet(lim-1) and wet(lim-2)
  end = w && (p == lim || !wp1) && ok;
}

// With dry != 0 the drying pass of Reset_states_vertical
// (support_funcs.cpp:177-186; dry = 1) or of Reset_states_horizontal
// (:125-137; dry = 2) is applied on the fly: a wet cell of its range (rows
// 2..N, columns 1..M; rows 1..N, columns 2..M) whose depth is at most H_TINH
// reads as dried (1) and is written so. Reading a neighbour's mask while
// its thread writes it is safe: the write turns 0 into 1 exactly when this
// test gives 1.
template <class R, int BATCH = 0>
__global__ void k_runs_flags(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int dry) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  int* seg_cnt = S.segcnt;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int i = blockIdx.y + 2;
  if (i > S.N || j > S.M) return;
  const int W = S.W, H = S.H, g = i * W + j;
  int* K = S.khouot;
  // every operand first (one round of memory latency): the masks, and with
  // dry the depths, of the cell and of its neighbours the run tests read
  // (all inside the array for rows 2..N, columns 2..M)
  const int qs[7] = {g, g - 1, g + 1, g - 2, g - W, g + W, g - 2 * W};
  int kk[7];
  R hh[7];
#pragma unroll
  for (int n = 0; n < 7; ++n) {
    kk[n] = K[qs[n]];
    hh[n] = dry ? S.Hmoi[qs[n]] : R(0);
  }
  const int ilo = dry == 2 ? 1 : 2, jlo = dry == 2 ? 2 : 1;
  auto mask = [&](int n, int qi, int qj) -> int {
    const int k = kk[n];
    if (dry && k == 0 && qi >= ilo && qi <= S.N && qj >= jlo && qj <= S.M && hh[n] <= c.H_TINH)
      return 1;
    return k;
  };
  if (dry) {
    const int k0 = mask(0, i, j);
    if (k0 != kk[0]) K[g] = k0;
    if (dry == 1 && j == 2) {  // column 1 is outside this grid
      const int k1 = mask(1, i, 1);
      if (k1 != kk[1]) K[g - 1] = k1;
    }
    if (dry == 2 && i == 2) {  // and so is row 1
      const int k4 = mask(4, 1, j);
      if (k4 != kk[4]) K[g - W] = k4;
    }
  }
  const bool w = mask(0, i, j) == 0;
  if (!w) return;
  // row i, position j, lim M
  {
    const bool wm1 = mask(1, i, j - 1) == 0, wp1 = mask(2, i, j + 1) == 0;
    const bool wm2 = mask(3, i, j - 2) == 0;
    bool st, en;
    run_flags(wm1, w, wp1, wm2, j, S.M, st, en);
    if (st) {
      const int s = atomicAdd(&seg_cnt[i], 1);
      if (s < SEG) S.daui[i * SEG + s] = j;
    }
    if (en) {
      const int s = atomicAdd(&seg_cnt[H + i], 1);
      if (s < SEG) S.cuoii[i * SEG + s] = j;
    }
  }
  // column j, position i, lim N
  {
    const bool wm1 = mask(4, i - 1, j) == 0, wp1 = mask(5, i + 1, j) == 0;
    const bool wm2 = mask(6, i - 2, j) == 0;
    bool st, en;
    run_flags(wm1, w, wp1, wm2, i, S.N, st, en);
    if (st) {
      const int s = atomicAdd(&seg_cnt[2 * H + j], 1);
      if (s < SEG) S.dauj[j * SEG + s] = i;
    }
    if (en) {
      const int s = atomicAdd(&seg_cnt[2 * H + W + j], 1);
      if (s < SEG) S.cuoij[j * SEG + s] = i;
    }
  }
}

__device__ __forceinline__ void sort_small(int* a, int n) {
  for (int x = 1; x < n; ++x) {
    const int v = a[x];
    int y = x - 1;
    while (y >= 0 && a[y] > v) {
      a[y + 1] = a[y];
      --y;
    }
    a[y + 1] = v;
  }
}

// One thread per line: order the claimed slots, set the counts, clear the
// counters for the next scan.
template <class R, int BATCH = 0>
__global__ void k_runs_sort(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  int* seg_cnt = S.segcnt;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int H = S.H, W = S.W;
  const int nrow = S.N - 1, ncol = S.M - 1;
  if (t >= nrow + ncol) return;
  int *dau, *cuoi, *moc, *cs, *ce;
  if (t < nrow) {
    const int i = t + 2;
    dau = S.daui + i * SEG;
    cuoi = S.cuoii + i * SEG;
    moc = S.moci + i;
    cs = seg_cnt + i;
    ce = seg_cnt + H + i;
  } else {
    const int j = t - nrow + 2;
    dau = S.dauj + j * SEG;
    cuoi = S.cuoij + j * SEG;
    moc = S.mocj + j;
    cs = seg_cnt + 2 * H + j;
    ce = seg_cnt + 2 * H + W + j;
  }
  int n = *cs;
  if (n > SEG || *ce != n) {
    atomicOr(S.err, DEV_SEG_OVERFLOW);
    n = min(n, SEG);
  }
  sort_small(dau, n);
  sort_small(cuoi, n);
  *moc = n;
  *cs = 0;
  *ce = 0;
}

template <class R>
__global__ void k_htuongdoi(StateT<R> S) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i = blockIdx.y + 1;
  if (i > S.N || j > S.M) return;
  const int W = S.W, p = i * W + j;
  S.Htdu[p] = (S.h[p - 1] + S.h[p] + S.z[p + W] + S.z[p]) * 0.5;
  S.Htdv[p] = (S.h[p - W] + S.h[p] + S.z[p + 1] + S.z[p]) * 0.5;
}

// preprocess_data with one CTA per side: the per-cell powers in parallel,
// each segment's sum in the reference's order by one thread (so the sums
// round as the reference's), the boundary-depth maximum by one thread.
// side: 0 up (column M), 1 down (column 2, node column 1), 2 left (row 2,
// node row 1), 3 right (row N).
template <class R>
__global__ void k_preprocess_sides(StateT<R> S, CoefT<R> c, double* p53) {
  const int side = blockIdx.x;
  const int W = S.W, M = S.M, N = S.N;
  const double dX = c.dX, ND = c.NANGDAY, ros = c.ros;
  const bool col = side < 2;
  const int loc = side == 0 ? M : (side == 3 ? N : 2);
  const int* moc = col ? S.mocj : S.moci;
  const int* dau = col ? S.dauj : S.daui;
  const int* cuoi = col ? S.cuoij : S.cuoii;
  double* hi = S.hi + (side == 0 ? 0 : side == 1 ? (N + 3) : side == 2 ? 2 * (N + 3) : 2 * (N + 3) + (M + 3));
  double* pw = p53 + side * (max(M, N) + 3);
  __shared__ double sums[SEG];
  const int nseg = moc[loc];
  for (int k = 0; k < nseg; ++k) {
    const int a = dau[loc * SEG + k], b = cuoi[loc * SEG + k];
    for (int p = a + threadIdx.x; p <= b; p += blockDim.x) {
      double v;
      if (side == 0) v = (S.h[p * W + M] + S.h[(p - 1) * W + M]) / 2.0 - ND;
      else if (side == 1) v = (S.h[p * W + 1] + S.h[(p - 1) * W + 1]) / 2.0 - ND;
      else if (side == 2) v = (S.h[1 * W + p] + S.h[1 * W + p - 1]) / 2.0 - ND;
      else v = (S.h[N * W + p] + S.h[N * W + p - 1]) / 2.0 - ND;
      hi[p] = v;
      pw[p] = pow(v, 5.0 / 3.0);
    }
  }
  __syncthreads();
  if (threadIdx.x < nseg) {
    const int k = threadIdx.x;
    double sum = 0;
    for (int p = dau[loc * SEG + k]; p <= cuoi[loc * SEG + k]; ++p) sum += pw[p];
    sums[k] = sum;
  }
  __syncthreads();
  for (int k = 0; k < nseg; ++k) {
    const int a = dau[loc * SEG + k], b = cuoi[loc * SEG + k];
    for (int p = a + threadIdx.x; p <= b; p += blockDim.x)
      hi[p] = pow(hi[p], 2.0 / 3.0) / (sums[k] * dX);
  }
  if (threadIdx.x == 0) {
    const double* hb = S.htaiz_bd;
    double mx;
    if (side == 0 || side == 1) {
      const int jj = side == 0 ? M : 2;
      mx = hb[2 * W + jj];
      for (int i = 3; i < N; ++i)
        if (hb[i * W + jj] > mx) mx = hb[i * W + jj];
    } else {
      const int ii = side == 2 ? 2 : N;
      mx = hb[ii * W + 2];
      for (int j = 3; j < M; ++j)
        if (hb[ii * W + j] > mx) mx = hb[ii * W + j];
    }
    S.hmax[side] = mx != 0 ? 1.0 / (ros * mx) : mx;
  }
}

// ------------------------------------------------------------- boundary
// The simulated time lives on the device so that a captured step replays
// unchanged: advanced by t += dT/2 per half-step (engine.cpp:66, 176).
// Update_Boundary_Value (support_funcs.cpp:682-728) at the device clock
// advanced by `half` (a half-step's time, or 0). t arrives through a float
// parameter in the reference (engine.cpp:22), hence the rounding. With half
// != 0 the last block to finish stores the advanced clock (clock[1] counts
// the blocks), after every block has read the old one.
//
// In the narrow-channel mode (S.chan) the series are not applied
// (update_boundary_at_t, engine.cpp:24-30); with S.chan == 2 the standing
// wave of boundary_up / boundary_down / boundary_left / boundary_right
// (support_funcs.cpp:366-478) is imposed instead: thread i takes row i of
// the up and down sides and column i of the left and right ones, each side
// over the first wet segment of its line (the right side from row 2's
// first start to row N's first end, as written there).
template <class R>
__device__ void channel_wave_cell(const StateT<R>& S, double dX, double dY, double t, int i) {
  const int M = S.M, N = S.N, W = S.W;
  const double PI_ = 3.14159265358979323846;
  const double ct = cos(2 * PI_ / 27.75 * t);
  if (S.mocj[M] > 0 && S.dauj[M * SEG] <= i && i <= S.cuoij[M * SEG]) {
    S.tz[i * W + M] = 0.01 * ct * cos(2 * (PI_ / 100) * (100 - dY / 2));
    S.tz[i * W + M + 1] = 0.01 * ct * cos(2 * (PI_ / 100) * (100 + dY / 2));
  }
  if (S.mocj[2] > 0 && S.dauj[2 * SEG] <= i && i <= S.cuoij[2 * SEG]) {
    if (S.bienQ[1]) {
      S.vbd[i] = 0;
    } else {
      S.tz[i * W + 2] = 0.01 * ct * cos(2 * (PI_ / 100) * dY / 2);
      S.tz[i * W + 1] = 0.01 * ct * cos(2 * (PI_ / 100) * (-dY) / 2);
    }
  }
  if (S.moci[2] > 0 && S.daui[2 * SEG] <= i && i <= S.cuoii[2 * SEG]) {
    if (S.bienQ[2]) {
      S.ubt[i] = 0;
    } else {
      S.tz[2 * W + i] = 0.01 * ct * cos(2 * (PI_ / 100) * dX / 2);
      S.tz[1 * W + i] = 0.01 * ct * cos(2 * (PI_ / 100) * (-dX) / 2);
    }
  }
  if (S.moci[2] > 0 && S.moci[N] > 0 && S.daui[2 * SEG] <= i && i <= S.cuoii[N * SEG]) {
    if (S.bienQ[3]) {
      S.ubp[i] = 0;
    } else {
      S.tz[N * W + i] = 0.01 * ct * cos(2 * (PI_ / 100) * (100 - dX / 2));
      S.tz[(N + 1) * W + i] = 0.01 * ct * cos(2 * (PI_ / 100) * (100 + dX / 2));
    }
  }
}

template <class R, int BATCH = 0>
__device__ __forceinline__ void boundary_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, double half) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const double dX = (double)c.dX, dY = (double)c.dY;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int M = S.M, N = S.N, W = S.W;
  const double t_new = S.clock[0] + half;
  if (half != 0) {
    __syncthreads();  // every thread of the block has read the clock
    if (threadIdx.x == 0 && atomicAdd(&S.clock[1], 1.0) == (double)(gridDim.x - 1)) {
      S.clock[0] = t_new;
      S.clock[1] = 0;
    }
  }
  if (i > M && i > N) return;
  const double t = (double)(float)t_new;
  if (S.chan) {
    if (S.chan == 2) channel_wave_cell(S, dX, dY, t, i);
    return;
  }
  // the host refuses steps past the series; the clamp keeps reads in bounds
  const int t1 = min(max((int)(t / 3600), 0), S.T - 2);
  const double t2h = (t - (double)(3600.0f * (float)t1)) / 3600.0f;
  const double t2f = (t - (3600.0 * t1)) / 3600.0;
  const double* hi_up = S.hi;
  const double* hi_down = hi_up + (N + 3);
  const double* hi_left = hi_down + (N + 3);
  const double* hi_right = hi_left + (M + 3);
  // every operand of the four sides first (one round of memory latency);
  // the indexed ones only where the index lies in their array
  int mo[4], d0[4], c0[4], bt[4];
  double bv0[4], bv1[4], cv0[4], cv1[4], hv[4], hb[4], hx[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const bool isU = s >= 2;
    const int loc = s == 0 ? M : (s == 3 ? N : 2);
    const int* moc = isU ? S.moci : S.mocj;
    const int* dau = isU ? S.daui : S.dauj;
    const int* cuoi = isU ? S.cuoii : S.cuoij;
    const double* hiv = s == 0 ? hi_up : (s == 1 ? hi_down : (s == 2 ? hi_left : hi_right));
    const int hlen = s < 2 ? N + 3 : M + 3;
    const int ii = isU ? loc : i, jj = isU ? i : loc;
    mo[s] = moc[loc];
    d0[s] = dau[loc * SEG];  // only segment 0 is matched (support_funcs.cpp:614-618)
    c0[s] = cuoi[loc * SEG];
    bt[s] = S.btype[s * SEG];
    bv0[s] = S.bc[s][t1];
    bv1[s] = S.bc[s][t1 + 1];
    cv0[s] = S.CC[s][t1];
    cv1[s] = S.CC[s][t1 + 1];
    hv[s] = i < hlen ? hiv[i] : 0.0;
    hb[s] = (ii < S.H && jj < W) ? S.htaiz_bd[ii * W + jj] : 0.0;
    hx[s] = S.hmax[s];
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const bool isU = s >= 2;
    const int loc = s == 0 ? M : (s == 3 ? N : 2);
    const int ext = s == 0 ? M + 1 : (s == 3 ? N + 1 : 1);
    R* barr = s == 0 ? S.vbt : (s == 1 ? S.vbd : (s == 2 ? S.ubt : S.ubp));
    if (mo[s] <= 0) continue;
    if (!(d0[s] <= i && i <= c0[s])) continue;
    const double val = bv0[s] * (1.0f - t2h) + bv1[s] * t2h;
    if (bt[s] == 2) {
      barr[i] = val * hv[s];
    } else {
      if (isU) {
        S.tz[loc * W + i] = val;
        S.tz[ext * W + i] = val;
      } else {
        S.tz[i * W + loc] = val;
        S.tz[i * W + ext] = val;
      }
    }
    if (bt[s] != 2) continue;
    const double cv = cv0[s] * (1.0 - t2f) + cv1[s] * t2f;
    const int ii = isU ? loc : i;
    const int jj = isU ? i : loc;
    S.FS[ii * W + jj] = cv * hb[s] * hx[s];
  }
}

// ------------------------------------------------------------ smoothing
// _normalize / update_buffer (support_funcs.cpp:761-808) into a complete
// array (su / sv): smoothed on the interior [2,N]x[2,M], the unsmoothed
// value elsewhere, i.e. t_u / t_v as they stand after update_buffer.
// Readers of the smoothed velocity use it directly and the half-step commit
// writes it back to t_u / t_v, u / v. hmoi != 0 (the last smoothing of
// half-step B, after the explicit u update that reads H_moi) also does
// update_h_moi and flags the columns (hmoi = 1) or rows (hmoi = 2) the
// wetting pass must visit.
// One thread smooths SMOOTH_ROWS consecutive rows of a column: the column's
// values and mask over those rows and the two around them are loaded once
// and shared between the rows, every operand before any arithmetic.
constexpr int SMOOTH_ROWS = 4;

// isU: t_u (else t_v); hmoi: with update_h_moi and the column flags. Both
// are template parameters: each launch compiles to its own variant.
// (ten CTAs per SM, eight for a batch: 3 us less per FP32 step on 2048x1024)
template <class R, int isU, int hmoi, int BATCH = 0>
__global__ void __launch_bounds__(128, BATCH ? 8 : 10)
    k_smooth_full(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  constexpr int RB = SMOOTH_ROWS;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * RB;
  if (j >= S.W) return;
  const int W = S.W, H = S.H, N = S.N, M = S.M;
  const R* val = isU ? S.tu : S.tv;
  R* out_arr = isU ? S.su : S.sv;
  const bool jin = j >= 2 && j <= M;
  // column j over rows i0-1 .. i0+RB (clamped to the array; the clamped
  // values are never used)
  R col[RB + 2];
  int kcol[RB + 2];
#pragma unroll
  for (int r = 0; r < RB + 2; ++r) {
    const int i = min(max(i0 - 1 + r, 0), H - 1);
    col[r] = val[i * W + j];
    kcol[r] = S.khouot[i * W + j];
  }
  // the row neighbours (j-1, j+1) of each row, interior cells only
  R sa[RB], sb[RB];
  int ka[RB], kb[RB];
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    const int i = i0 + r;
    sa[r] = sb[r] = 0;
    ka[r] = kb[r] = 0;
    if (i >= 2 && i <= N && jin) {
      const int g = i * W + j;
      sa[r] = val[g - 1];
      sb[r] = val[g + 1];
      if (isU) {
        ka[r] = S.khouot[g - 1];
        kb[r] = S.khouot[g + 1];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < RB; ++r) {
    const int i = i0 + r;
    if (i >= H) break;
    const int g = i * W + j;
    if (hmoi && i >= 1 && i <= N + 1 && j >= 1 && j <= M) {
      const int kh = kcol[r + 1];
      if (i <= N && kh == 0) S.Hmoi[g] = S.htaiz[g] + S.tz[g];
      if (kh == 1) {
        if (hmoi == 2) {
          if (i <= N) S.rowflag[i] = 1;
        } else {
          S.colflag[j] = 1;
        }
      }
    }
    const R vg = col[r + 1];
    R out = vg;
    if (i >= 2 && i <= N && jin && vg != 0) {
      // u: the close neighbours are the rows above and below, the far ones
      // (counted where wet) the columns; v the other way round
      const R a = isU ? col[r] : sa[r], b = isU ? col[r + 2] : sb[r];
      const R l = isU ? sa[r] : col[r], rr = isU ? sb[r] : col[r + 2];
      const int kl = isU ? ka[r] : kcol[r], kr = isU ? kb[r] : kcol[r + 2];
      int count = 2;
      R nb = a + b;
      if (kl == 0) {
        nb += l;
        count++;
      }
      if (kr == 0) {
        nb += rr;
        count++;
      }
      out = out * c.heso + (1 - c.heso) * nb / count;
    }
    out_arr[g] = out;
  }
}

// ---------------------------------------------------- explicit updates
__device__ __forceinline__ bool find_seg(const int* dau, const int* cuoi, int n, int pos, int& first,
                                         int& last) {
  for (int k = 0; k < n; ++k) {
    if (dau[k] <= pos && pos <= cuoi[k]) {
      first = dau[k];
      last = cuoi[k];
      return true;
    }
  }
  return false;
}

// vSolver driven by solveV (UVZSolver_multithread.cpp:607-663, 961-978);
// the cell's arithmetic is v_new (explicit.cuh).
template <class R, int BATCH = 0>
__device__ __forceinline__ void solve_v_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  // the block's cells share one row: its segment table goes to shared memory
  __shared__ int s_first[SEG], s_last[SEG];
  __shared__ int s_n;
  const int col = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int row = blockIdx.y + 2;
  const bool ok = row <= S.N && col <= S.M;
  const int g = row * S.W + col;
  // every operand, in bounds for rows 2..N and columns 2..M, is loaded
  // with the segment table, before the lookup that decides whether the
  // cell is updated: one round of memory latency
  VOps<R> o;
  if (ok) o = v_ops(S, S.su, g);  // t_u after its smoothing
  if (threadIdx.x < SEG) {
    s_first[threadIdx.x] = S.daui[row * SEG + threadIdx.x];
    s_last[threadIdx.x] = S.cuoii[row * SEG + threadIdx.x];
  }
  if (threadIdx.x == 0) s_n = S.moci[row];
  __syncthreads();
  if (!ok) return;
  int first, last;
  if (!find_seg(s_first, s_last, s_n, col, first, last)) return;
  if (first >= last || col >= last || col < first) return;
  S.tv[g] = v_new(o, c);
}

// uSolver driven by solveU (UVZSolver_multithread.cpp:724-795, 938-959);
// the cell's arithmetic is u_new (explicit.cuh).
template <class R, int BATCH = 0>
__device__ __forceinline__ void solve_u_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int col = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int row = blockIdx.y + 1;
  if (row > S.N || col > S.M) return;
  const int ij = row * S.W + col;
  // every operand is loaded before the segment lookup (all in bounds for
  // rows 1..N, columns 2..M), so both take one round of memory latency
  const UOps<R> o = u_ops(S, S.sv, ij);  // t_v after its smoothing
  int first, last;
  if (!find_seg(S.dauj + col * SEG, S.cuoij + col * SEG, S.mocj[col], row, first, last)) return;
  if (first > last || row < first - 1 || row >= last) return;
  S.tu[ij] = u_new(o, c);
}

// update_margin_elem_V (UVZSolver_multithread.cpp:1018-1060), one row per
// thread.
template <class R, int BATCH = 0>
__global__ void k_margin_v(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (i > S.N) return;
  margin_v(S, (double)c.NANGDAY, i);
}

// update_margin_elem_U (UVZSolver_multithread.cpp:980-1016), one column per
// thread.
template <class R, int BATCH = 0>
__global__ void k_margin_u(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (j > S.M) return;
  margin_u(S, (double)c.NANGDAY, j);
}

// ------------------------------------------------------ fused commits
// Find_VTH (sediment_transport.cpp:575-602) and hesoK (:539-573) of cell
// (i, j) from the committed values the commit holds: tu, tv of the cell,
// tu_up = t_u(i-1, j), tv_left = t_v(i, j-1), H_moi, the bed depths h of the
// cell, of (i, j-1) and of (i-1, j), and the new Htdu, Htdv. Rows 1..vth_hi
// (the sediment launch shape: N after half-step A, N-1 after B), VTH from
// row and column 2.
// Returns the speed stored at (i, j) (0 where none is, i or j below 2).
template <class R>
__device__ __forceinline__ R vth_heso_cell(const StateT<R>& S, const CoefT<R>& c, int i, int j,
                                           int g, R tu, R tv, R tu_up, R tv_left, R Hm,
                                           double ht, double hp, double hl, double hup, R Hu,
                                           R Hv) {
  R vthv = 0;
  if (i >= 2 && j >= 2) {
    if ((ht > c.NANGDAY) && (Hm > c.H_TINH)) {
      const R ut = (tu + tu_up) * R(0.5);
      const R vt = (tv + tv_left) * R(0.5);
      vthv = sqrt(ut * ut + vt * vt);
    }
    S.VTH[g] = vthv;
  }
  if (Hu > 0) {
    const R Cz = 18 * log(12 * Hu / c.Ks);
    const R k = R(5.93) * c.sqrt_g * R(hl + hp) * R(0.25) * fabs(tu) / Cz;
    S.Kx[g] = fmin(R(100), fmax(R(5), k));
  }
  if (Hv > 0) {
    const R Cz = 18 * log(12 * Hv / c.Ks);
    const R k = R(5.93) * c.sqrt_g * R(hup + hp) * R(0.25) * fabs(tv) / Cz;
    S.Ky[g] = fmin(R(100), fmax(R(5), k));
  }
  return vthv;
}

// Half-step A commit: update_h_moi (support_funcs.cpp:71-86) on [1,N]x[1,M],
// update_uvz (:732-759) on [0,N]x[0,M] and Htuongdoi (:346-362) on
// [1,N]x[1,M] in one pass. Htuongdoi reads the committed z of the
// neighbour: t_z where it was committed, z where it never is (row N+1,
// column M+1). With vth_hi > 0 (the concentration step follows) also
// Find_VTH + hesoK on rows 1..vth_hi: nothing between this commit and the
// concentration sweep changes what they read.
template <class R, int BATCH = 0>
__device__ __forceinline__ void commit_a_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int vth_hi) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (i > S.N || j > S.M) return;
  const int W = S.W, g = i * W + j;
  const bool in = i >= 1 && j >= 1;
  const bool vth = in && i <= vth_hi;
  // every operand before the first store (one round of memory latency);
  // nothing this kernel stores is read by another of its threads
  const double tz = S.tz[g];
  const int kh = S.khouot[g];
  const double ht = S.htaiz[g];
  const R hm_old = S.Hmoi[g];
  const R tu = S.su[g], tv = S.sv[g];  // t_u, t_v after their smoothing
  const double zd = (i + 1 <= S.N) ? S.tz[g + W] : S.z[g + W];
  const double zr = (j + 1 <= S.M) ? S.tz[g + 1] : S.z[g + 1];
  const double hp = S.h[g];
  const double hl = in ? S.h[g - 1] : 0.0, hup = in ? S.h[g - W] : 0.0;
  // the committed t_u(i-1, j), t_v(i, j-1) are the smoothed values there
  const R tu_up = vth ? S.su[g - W] : R(0), tv_left = vth ? S.sv[g - 1] : R(0);
  R Hm = 0;
  if (in) {
    if (kh == 0) {
      Hm = ht + tz;
      S.Hmoi[g] = Hm;
    } else if (vth) {
      Hm = hm_old;
    }
  }
  S.tu[g] = tu;
  S.tv[g] = tv;
  S.z[g] = tz;
  S.u[g] = tu * (1 - c.kenhhepd);
  S.v[g] = tv * (1 - c.kenhhepng);
  canary(S.err, (double)tu, (double)tv, tz);
  if (in) {
    const R Hu = (hl + hp + zd + tz) * 0.5;
    const R Hv = (hup + hp + zr + tz) * 0.5;
    S.Htdu[g] = Hu;
    S.Htdv[g] = Hv;
    if (vth) vth_heso_cell(S, c, i, j, g, tu, tv, tu_up, tv_left, Hm, ht, hp, hl, hup, Hu, Hv);
  }
}

// The wetting loop of Reset_states_vertical (support_funcs.cpp:160-175),
// sequential along i, on flagged columns only.
template <class R, int BATCH = 0>
__global__ void k_wetting(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  int* colflag = S.colflag;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (j > S.M) return;
  if (!colflag[j]) return;
  colflag[j] = 0;
  const int off = S.W, N = S.N;
  double* tz = S.tz;
  R* Hm = S.Hmoi;
  int* kh = S.khouot;
  for (int i = 2; i <= N; ++i) {
    if (tz[i * off + j] > S.z[i * off + j]) {
      if (kh[(i - 1) * off + j] == 1) {
        tz[(i - 1) * off + j] = tz[i * off + j];
        Hm[(i - 1) * off + j] = S.htaiz[(i - 1) * off + j] + tz[i * off + j];
        kh[(i - 1) * off + j] = 0;
        S.FS[(i - 1) * off + j] = S.FS[i * off + j];
      }
      if (kh[(i + 1) * off + j] == 1) {
        tz[(i + 1) * off + j] = tz[i * off + j];
        Hm[(i + 1) * off + j] = S.htaiz[(i + 1) * off + j] + tz[i * off + j];
        kh[(i + 1) * off + j] = 0;
        S.FS[(i + 1) * off + j] = S.FS[i * off + j];
      }
    }
  }
}

// The wetting loop of Reset_states_horizontal (support_funcs.cpp:103-120),
// sequential along j, on flagged rows 1..N only.
template <class R, int BATCH = 0>
__global__ void k_wetting_rows(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  int* rowflag = S.rowflag;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > S.N) return;
  if (!rowflag[i]) return;
  rowflag[i] = 0;
  const int M = S.M;
  const size_t r = (size_t)i * S.W;
  double* tz = S.tz;
  R* Hm = S.Hmoi;
  int* kh = S.khouot;
  for (int j = 2; j <= M; ++j) {
    if (tz[r + j] > S.z[r + j]) {
      if (kh[r + j - 1] == 1) {
        tz[r + j - 1] = tz[r + j];
        Hm[r + j - 1] = S.htaiz[r + j - 1] + tz[r + j];
        kh[r + j - 1] = 0;
        S.FS[r + j - 1] = S.FS[r + j];
      }
      if (kh[r + j + 1] == 1) {
        tz[r + j + 1] = tz[r + j];
        Hm[r + j + 1] = S.htaiz[r + j + 1] + tz[r + j];
        kh[r + j + 1] = 0;
        S.FS[r + j + 1] = S.FS[r + j];
      }
    }
  }
}

// Half-step B commit: the drying loop of Reset_states_vertical (:177-187,
// independent per cell), update_uvz and Htuongdoi. A drying cell (i,j)
// zeroes t_u at (i-1,j),(i,j) and t_v at (i,j-1),(i,j); each cell here reads
// its own test and those of (i+1,j) and (i,j+1).
//
// With vth_hi > 0 also Find_VTH + hesoK on rows 1..vth_hi, as in
// k_commit_a: the segment scan and the boundary interpolation that follow
// change none of their operands. The committed t_u(i-1, j) and t_v(i, j-1)
// are rebuilt here from the same drying tests their own threads make.
//
// HORIZ: the drying loop of Reset_states_horizontal instead (:125-137,
// rows 1..N, columns 2..M), in the first half-step.
//
// qb != 0 (the bed change follows this step's concentration j-sweep): also
// Calculate_Qb (qb_cell) on rows 2..N, columns 2..M, from the committed
// velocities, the speed, the mask after the drying pass and H_moi; nothing
// between this pass and BedLoad changes them. On row N the speed is the
// first half-step's (its hesoK launch shape never reaches row N).
template <class R, int HORIZ, int BATCH = 0>
__device__ __forceinline__ void commit_b_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int vth_hi, int qb) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (i > S.N || j > S.M) return;
  const int W = S.W, g = i * W + j;
  const bool in = i >= 1 && j >= 1;
  const bool vth = in && i <= vth_hi;
  const bool qbc = qb && i >= 2 && j >= 2;
  const bool nbr = vth || qbc;  // the committed t_u(i-1, j), t_v(i, j-1) are needed
  // every operand before the first store (one round of memory latency);
  // nothing this kernel stores is read by another of its threads. A cell
  // dries when it is wet with H_moi at most H_TINH (rows 2..N, columns 1..M;
  // rows 1..N, columns 2..M with HORIZ).
  auto in_dry = [&](int ii, int jj) {
    return HORIZ ? (ii >= 1 && ii <= S.N && jj >= 2 && jj <= S.M)
                 : (ii >= 2 && ii <= S.N && jj >= 1 && jj <= S.M);
  };
  const bool c0 = in_dry(i, j), cd = in_dry(i + 1, j), cr = in_dry(i, j + 1);
  const bool cu = nbr && in_dry(i - 1, j), cl = nbr && in_dry(i, j - 1);
  const int k0 = c0 ? S.khouot[g] : 1, kd = cd ? S.khouot[g + W] : 1, kr = cr ? S.khouot[g + 1] : 1;
  const int ku = cu ? S.khouot[g - W] : 1, kl = cl ? S.khouot[g - 1] : 1;
  const R h0 = c0 ? S.Hmoi[g] : R(0), hd = cd ? S.Hmoi[g + W] : R(0), hr = cr ? S.Hmoi[g + 1] : R(0);
  const R hu = cu ? S.Hmoi[g - W] : R(0), hl_ = cl ? S.Hmoi[g - 1] : R(0);
  const double su = S.su[g], sv = S.sv[g];
  const double tz = S.tz[g];
  const double zd = (i + 1 <= S.N) ? S.tz[g + W] : S.z[g + W];
  const double zr = (j + 1 <= S.M) ? S.tz[g + 1] : S.z[g + 1];
  const double hp = S.h[g];
  const double hl = in ? S.h[g - 1] : 0.0, hup = in ? S.h[g - W] : 0.0;
  const double ht = vth ? S.htaiz[g] : 0.0;
  const R hm = (vth || qbc) ? S.Hmoi[g] : R(0);
  const R su_up = nbr ? S.su[g - W] : R(0), sv_left = nbr ? S.sv[g - 1] : R(0);
  const R fw = qbc ? S.Fw[g] : R(0);
  const R vth_old = (qbc && !vth) ? S.VTH[g] : R(0);
  const bool d0 = c0 && k0 == 0 && h0 <= c.H_TINH;
  const bool ddown = cd && kd == 0 && hd <= c.H_TINH;
  const bool dright = cr && kr == 0 && hr <= c.H_TINH;
  // t_u, t_v after their smoothing, zeroed by the drying pass
  double tu = su, tv = sv;
  if (d0 || ddown) tu = 0;
  if (d0 || dright) tv = 0;
  S.tu[g] = tu;
  S.tv[g] = tv;
  if (d0) S.FS[g] = 0;  // khouot is set by the segment scan after this pass
  S.z[g] = tz;
  S.u[g] = tu * (1 - c.kenhhepd);
  S.v[g] = tv * (1 - c.kenhhepng);
  canary(S.err, tu, tv, tz);
  if (in) {
    const R Hu = (hl + hp + zd + tz) * 0.5;
    const R Hv = (hup + hp + zr + tz) * 0.5;
    S.Htdu[g] = Hu;
    S.Htdv[g] = Hv;
    if (nbr) {
      // t_u(i-1, j) is zeroed when (i-1, j) or (i, j) dries, t_v(i, j-1)
      // when (i, j-1) or (i, j) does
      const bool dup = cu && ku == 0 && hu <= c.H_TINH;
      const bool dleft = cl && kl == 0 && hl_ <= c.H_TINH;
      const R tu_up = (dup || d0) ? R(0) : su_up;
      const R tv_left = (dleft || d0) ? R(0) : sv_left;
      R vthv = vth_old;
      if (vth) vthv = vth_heso_cell(S, c, i, j, g, R(tu), R(tv), tu_up, tv_left, hm, ht, hp, hl, hup, Hu, Hv);
      // the mask after this pass's drying (the segment scan writes it)
      if (qbc) qb_cell(S, c, i, j, vthv, d0 ? 1 : k0, hm, fw, R(tu), tu_up, R(tv), tv_left);
    }
  }
}

// The drying cells' mask (khouot = 1), written after k_commit_b has read
// every neighbour's test.
// ------------------------------------------------------------- launchers
static inline dim3 grid2(int nx, int ny, int bx) { return dim3(cdiv(nx, bx), ny); }

// Launches a step kernel for one scenario (ks, b.n == 0) or for every
// member of a batch (kb, grid z = members).
// Entry points of the passes above: the single-scenario kernels unbounded,
// the batch ones (suffix _b) under HYD_CELL_BOUNDS. A bound changes ptxas's
// register choice even where it does not bind, so the two are separate
// kernels.
template <class R, int BATCH = 0>
__global__ void k_boundary(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, double half) {
  boundary_cells<R, BATCH>(S_arg, c_arg, b_arg, half);
}
template <class R>
__global__ void HYD_CELL_BOUNDS k_boundary_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, double half) {
  boundary_cells<R, 1>(S_arg, c_arg, b_arg, half);
}

template <class R, int BATCH = 0>
__global__ void k_solve_v(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  solve_v_cells<R, BATCH>(S_arg, c_arg, b_arg);
}
template <class R>
__global__ void HYD_CELL_BOUNDS k_solve_v_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  solve_v_cells<R, 1>(S_arg, c_arg, b_arg);
}

template <class R, int BATCH = 0>
__global__ void k_solve_u(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  solve_u_cells<R, BATCH>(S_arg, c_arg, b_arg);
}
template <class R>
__global__ void HYD_CELL_BOUNDS k_solve_u_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  solve_u_cells<R, 1>(S_arg, c_arg, b_arg);
}

template <class R, int BATCH = 0>
__global__ void k_commit_a(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int vth_hi) {
  commit_a_cells<R, BATCH>(S_arg, c_arg, b_arg, vth_hi);
}
template <class R>
__global__ void HYD_CELL_BOUNDS k_commit_a_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int vth_hi) {
  commit_a_cells<R, 1>(S_arg, c_arg, b_arg, vth_hi);
}

// (the single-scenario second commit under the bound too: 66 -> 64 registers
// in FP64, eight CTAs per SM against seven, 4 us less per step on 2048x1024;
// the bed load so bounded was 3 us slower)
template <class R, int HORIZ, int BATCH = 0>
__global__ void HYD_CELL_BOUNDS k_commit_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int vth_hi,
                                           int qb) {
  commit_b_cells<R, HORIZ, BATCH>(S_arg, c_arg, b_arg, vth_hi, qb);
}
template <class R, int HORIZ>
__global__ void HYD_CELL_BOUNDS k_commit_b_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg, int vth_hi, int qb) {
  commit_b_cells<R, HORIZ, 1>(S_arg, c_arg, b_arg, vth_hi, qb);
}

template <class R, class KS, class KB, class... A>
static void launch2(KS ks, KB kb, dim3 g, int bs, cudaStream_t st, const StateT<R>& S,
                    const CoefT<R>& c, const Batch<R>& b, A... a) {
  if (b.n > 0) {
    g.z = (unsigned)b.n;
    kb<<<g, bs, 0, st>>>(S, c, b, a...);
  } else {
    ks<<<g, bs, 0, st>>>(S, c, b, a...);
  }
}
#define HYD_K2(name, ...) name<__VA_ARGS__, 0>, name<__VA_ARGS__, 1>
// the same for the passes with separate batch entry points (name_b)
#define HYD_K2B(name, ...) name<__VA_ARGS__, 0>, name##_b<__VA_ARGS__>

template <class R>
void launch_init(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st) {
  k_onetime_init<<<dim3(cdiv(S.W, 128), S.H), 128, 0, st>>>(S, c);
  launch_find_limits(S, c, false, st, nullptr);
  k_htuongdoi<<<grid2(S.M, S.N, 128), 128, 0, st>>>(S);
  // the per-side scratch of the powers: the line-solver scratch is free here
  k_preprocess_sides<<<4, 256, 0, st>>>(S, c, reinterpret_cast<double*>(S.lscratch));
}

template <class R>
void launch_preprocess(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st) {
  k_preprocess_sides<<<4, 256, 0, st>>>(S, c, reinterpret_cast<double*>(S.lscratch));
}

template <class R>
void launch_boundary(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st) {
  launch2(HYD_K2B(k_boundary, R), dim3(cdiv(max(S.M, S.N), 128)), 128, st, S, c, Batch<R>{}, 0.0);
}

template <class R>
void launch_scan_segments(const StateT<R>& S, const CoefT<R>& c, bool dry, cudaStream_t st,
                          const Batch<R>& b) {
  launch2(HYD_K2(k_runs_flags, R), grid2(S.M - 1, S.N - 1, 128), 128, st, S, c, b, dry ? 1 : 0);
  launch2(HYD_K2(k_runs_sort, R), dim3(cdiv(S.N + S.M - 2, 128)), 128, st, S, c, b);
}

template <class R>
void launch_find_limits(const StateT<R>& S, const CoefT<R>& c, bool dry, cudaStream_t st,
                        Trace* tr, const Batch<R>& b) {
  launch2(HYD_K2(k_interp_fs_rows, R), dim3(cdiv(S.M, 128), 2), 128, st, S, c, b);
  launch2(HYD_K2(k_interp_fs_col, R), dim3(cdiv(S.M, 128)), 128, st, S, c, b);
  launch_scan_segments(S, c, dry, st, b);
  if (tr) tr->launches += 4;
}

template <class R>
void launch_half_x(const StateT<R>& S, const CoefT<R>& c, bool sed, cudaStream_t st, Trace* tr,
                   const Batch<R>& b) {
  const dim3 cells(cdiv(S.M - 1, 128), S.N - 1);
  const dim3 smooth(cdiv(S.W, 128), cdiv(S.H, SMOOTH_ROWS));
  const dim3 commit(cdiv(S.M + 1, 128), S.N + 1);
  launch2(HYD_K2B(k_boundary, R), dim3(cdiv(max(S.M, S.N), 128)), 128, st, S, c, b, 0.5 * (double)c.dT);
  if (tr) tr->mark(st, PH_BOUNDARY_X, 1);
  if (tr) tr->kbegin(st, KS_SWEEP_X);
  const int nx = launch_sweep(S, c, 0, st, b);
  if (tr) tr->kend(st, KS_SWEEP_X);
  if (tr) tr->mark(st, PH_SWEEP_X, nx);
  // smoothing of t_u into su, explicit v from it, margins, smoothing of t_v
  // into sv; k_commit_a writes both back (Normalize/update_buffer pairs,
  // engine.cpp:109-124)
  launch2(HYD_K2(k_smooth_full, R, 1, 0), smooth, 128, st, S, c, b);
  launch2(HYD_K2B(k_solve_v, R), cells, 128, st, S, c, b);
  launch2(HYD_K2(k_margin_v, R), dim3(cdiv(S.N - 1, 128)), 128, st, S, c, b);
  if (S.reset_h) {
    // wetting and drying along rows (Reset_states_horizontal after
    // update_h_moi): the smoothing of t_v also does update_h_moi and flags
    // the rows holding a dried cell, the rows' wetting runs on those, the
    // drying per cell in the commit, the mask is written by the segment
    // scan (the mask can change, so the tables are rescanned)
    launch2(HYD_K2(k_smooth_full, R, 0, 2), smooth, 128, st, S, c, b);
    if (tr) tr->mark(st, PH_EXPLICIT_V, 4);
    launch2(HYD_K2(k_wetting_rows, R), dim3(cdiv(S.N, 128)), 128, st, S, c, b);
    launch2(HYD_K2B(k_commit_b, R, 1), commit, 128, st, S, c, b, sed ? S.N : 0, 0);
    launch2(HYD_K2(k_interp_fs_rows, R), dim3(cdiv(S.M, 128), 2), 128, st, S, c, b);
    launch2(HYD_K2(k_interp_fs_col, R), dim3(cdiv(S.M, 128)), 128, st, S, c, b);
    launch2(HYD_K2(k_runs_flags, R), grid2(S.M - 1, S.N - 1, 128), 128, st, S, c, b, 2);
    launch2(HYD_K2(k_runs_sort, R), dim3(cdiv(S.N + S.M - 2, 128)), 128, st, S, c, b);
    if (tr) tr->mark(st, PH_COMMIT_X, 6);
    return;
  }
  launch2(HYD_K2(k_smooth_full, R, 0, 0), smooth, 128, st, S, c, b);
  if (tr) tr->mark(st, PH_EXPLICIT_V, 4);
  // update_h_moi + update_uvz + Htuongdoi; the wet/dry mask does not change
  // in this half-step, so the segment tables are not rescanned, only the
  // boundary concentration is interpolated (support_funcs.cpp:255-258, 311)
  // with sed, also Find_VTH + hesoK of the concentration step (rows to N)
  launch2(HYD_K2B(k_commit_a, R), commit, 128, st, S, c, b, sed ? S.N : 0);
  launch2(HYD_K2(k_interp_fs_rows, R), dim3(cdiv(S.M, 128), 2), 128, st, S, c, b);
  launch2(HYD_K2(k_interp_fs_col, R), dim3(cdiv(S.M, 128)), 128, st, S, c, b);
  if (tr) tr->mark(st, PH_COMMIT_X, 3);
}

template <class R>
void launch_half_y(const StateT<R>& S, const CoefT<R>& c, bool sed, cudaStream_t st, Trace* tr,
                   const Batch<R>& b, bool qb) {
  const dim3 smooth(cdiv(S.W, 128), cdiv(S.H, SMOOTH_ROWS));
  const dim3 commit(cdiv(S.M + 1, 128), S.N + 1);
  launch2(HYD_K2B(k_boundary, R), dim3(cdiv(max(S.M, S.N), 128)), 128, st, S, c, b, (double)c.dT * 0.5);
  if (tr) tr->mark(st, PH_BOUNDARY_Y, 1);
  if (tr) tr->kbegin(st, KS_SWEEP_Y);
  const int ny = launch_sweep(S, c, 1, st, b);
  if (tr) tr->kend(st, KS_SWEEP_Y);
  if (tr) tr->mark(st, PH_SWEEP_Y, ny);
  launch2(HYD_K2(k_smooth_full, R, 0, 0), smooth, 128, st, S, c, b);
  launch2(HYD_K2B(k_solve_u, R), dim3(cdiv(S.M - 1, 128), S.N), 128, st, S, c, b);
  launch2(HYD_K2(k_margin_u, R), dim3(cdiv(S.M - 1, 128)), 128, st, S, c, b);
  // with update_h_moi and the wetting pass's column flags
  launch2(HYD_K2(k_smooth_full, R, 1, 1), smooth, 128, st, S, c, b);
  if (tr) tr->mark(st, PH_EXPLICIT_U, 4);
  // update_h_moi, Reset_states_vertical (wetting on flagged columns, drying
  // per cell), update_uvz, Htuongdoi, then the segment tables
  launch2(HYD_K2(k_wetting, R), dim3(cdiv(S.M, 128)), 128, st, S, c, b);
  // with sed, also Find_VTH + hesoK (rows to N-1: the launch shape of
  // engine.cpp:259-260 never reaches row N)
  // with qb, also Calculate_Qb of the bed change that follows this step's
  // concentration j-sweep
  launch2(HYD_K2B(k_commit_b, R, 0), commit, 128, st, S, c, b, sed ? S.N - 1 : 0,
          qb && S.N >= 5 ? 1 : 0);
  // the drying mask is written by the segment scan (k_runs_flags, dry)
  launch_find_limits(S, c, true, st, tr, b);
  if (tr) tr->mark(st, PH_COMMIT_Y, 2);
}

#define HYD_HYDRO_INST(R)                                                                  \
  template void launch_init<R>(const StateT<R>&, const CoefT<R>&, cudaStream_t);         \
  template void launch_preprocess<R>(const StateT<R>&, const CoefT<R>&, cudaStream_t);   \
  template void launch_boundary<R>(const StateT<R>&, const CoefT<R>&, cudaStream_t);    \
  template void launch_scan_segments<R>(const StateT<R>&, const CoefT<R>&, bool,         \
                                        cudaStream_t, const Batch<R>&);                   \
  template void launch_find_limits<R>(const StateT<R>&, const CoefT<R>&, bool, cudaStream_t, \
                                      Trace*, const Batch<R>&);                           \
  template void launch_half_x<R>(const StateT<R>&, const CoefT<R>&, bool, cudaStream_t, Trace*, \
                                 const Batch<R>&);                                        \
  template void launch_half_y<R>(const StateT<R>&, const CoefT<R>&, bool, cudaStream_t, Trace*, \
                                 const Batch<R>&, bool);
HYD_HYDRO_INST(double)
HYD_HYDRO_INST(float)

}  // namespace hyd
