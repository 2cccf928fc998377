// sediment.cu -- suspended-sediment concentration step on the GPU.
//
// Kernels (reference kernel each one replaces in brackets):
//   Find_VTH + hesoK [sediment_transport.cpp:575-602, 539-573] run in the
//                  hydraulic commits (hydro.cu: k_commit_a, k_commit_b)
//   the sweeps     [Scan_FSj/Scan_FSi + tridiagSolver + FSj/FSi_extract_
//                   solution, :51-349, 604-651]: the partitioned line solver
//                   with FSGen (sweep.cu), cell rows in sediment_cell.cuh
//   k_update_fs    [Update_FS, :654-663]
//   Calculate_Qb   [:352-434] runs in the second commit (hydro.cu k_commit_b)
//   k_bed_load     [_bed_load / BedLoad, :436-537, :664-673]
#include "common.cuh"
#include "hydro.cuh"
#include "sediment_cell.cuh"

namespace hyd {

// ---- bed change: Calculate_Qb (sediment_transport.cpp:352-434, qb_cell in
// sediment_cell.cuh) runs in the second half-step's commit (k_commit_b, with
// the values that pass holds), _bed_load / BedLoad (:436-537, :664-673) here;
// the reference never launches either (engine.cpp:290-293). Read as intended
// where the code cannot be meant literally: t_u[pos] > 0 in the downwind test
// (:479).
// _bed_load on rows 3..N-2 (BedLoad with the j-sweep's range,
// engine.cpp:292), cells of the row's wet segments of at least 3 cells.
template <class R, int BATCH = 0>
__device__ __forceinline__ void bed_load_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  __shared__ int s_first[SEG], s_last[SEG];
  __shared__ int s_n;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int i = blockIdx.y + 3;
  if (threadIdx.x < SEG) {
    s_first[threadIdx.x] = S.daui[i * SEG + threadIdx.x];
    s_last[threadIdx.x] = S.cuoii[i * SEG + threadIdx.x];
  }
  if (threadIdx.x == 0) s_n = S.moci[i];
  __syncthreads();
  if (i >= S.N - 1 || j > S.M) return;
  const int w = S.W, pos = i * w + j, M = S.M, N = S.N;
  const int* kh = S.khouot;
  const R *Qbx = S.Qbx, *Qby = S.Qby, *FS = S.FS;
  // every operand (all in bounds for rows 3..N-2, columns 2..M) before the
  // segment lookup and the upwind tests that choose among them: one round
  // of memory latency
  const int kN = kh[pos - w], kS = kh[pos + w], kN2 = kh[pos - 2 * w], kS2 = kh[pos + 2 * w];
  const int kW = kh[pos - 1], kE = kh[pos + 1], kW2 = kh[pos - 2], kE2 = kh[pos + 2];
  const R tu = S.tu[pos], tv = S.tv[pos];
  const R qx0 = Qbx[pos], qxN = Qbx[pos - w], qxS = Qbx[pos + w], qxN2 = Qbx[pos - 2 * w],
          qxS2 = Qbx[pos + 2 * w];
  const R qy0 = Qby[pos], qyW = Qby[pos - 1], qyE = Qby[pos + 1], qyW2 = Qby[pos - 2],
          qyE2 = Qby[pos + 2];
  const R fs = FS[pos], fN = FS[pos - w], fS = FS[pos + w], fW = FS[pos - 1], fE = FS[pos + 1];
  const R hu0 = S.Htdu[pos], huN = S.Htdu[pos - w], kx0 = S.Kx[pos], kxN = S.Kx[pos - w];
  const R hv0 = S.Htdv[pos], hvW = S.Htdv[pos - 1], ky0 = S.Ky[pos], kyW = S.Ky[pos - 1];
  const R Hm = S.Hmoi[pos], vth = S.VTH[pos];
  const R fw = S.ketdinh ? S.Fw[pos] : R(0);
  int first = 0, last = 0;
  for (int k = 0; k < s_n; ++k)
    if (s_first[k] <= j && j <= s_last[k]) {
      first = s_first[k];
      last = s_last[k];
      break;
    }
  if (last - first < 2 || j < first || j > last) return;
  R p = 0, q = 0;
  if (kN == 1) {
    if (tu < 0) p = (-3 * qx0 + 4 * qxS - qxS2) * c.r_dX2;
  } else {
    if (kS == 1) {
      if (tu > 0) p = (3 * qx0 - 4 * qxN + qxN2) * c.r_dX2;
    } else {
      p = (qxS - qxN) * c.r_dX2;
    }
  }
  if (kW == 1) {
    if (tv < 0) q = (-3 * qy0 + 4 * qyE - qyE2) * c.r_dY2;
  } else {
    if (kE == 1) {
      if (tv > 0) q = (3 * qy0 - 4 * qyW + qyW2) * c.r_dY2;
    } else {
      q = (qyE - qyW) * c.r_dY2;
    }
  }
  R tH = p + q;
  p = fS - fs;
  if ((kS2 == 1 || kN == 1) && (i < N)) p = 0;
  q = fs - fN;
  if ((i > 2) && (kN2 == 1 || kS == 1)) q = 0;
  p = c.r_dXbp * (hu0 * kx0 * p - huN * kxN * q);
  tH = tH + p;
  p = fE - fs;
  if (((last < M) && (kW == 1 || kE2 == 1)) || (last == M && (kW == 1))) p = 0;
  q = fs - fW;
  if (((first > 2) && (kW2 == 1 || kE == 1)) || (first == 2 && kE == 1)) q = 0;
  p = c.r_dYbp * (hv0 * ky0 * p - hvW * kyW * q);
  tH = tH + p;
  const R cc = 18 * log(12 * Hm / c.Ks);
  const R Uf = c.sqrt_g * fabs(vth) / cc;
  const R om = 1 - fs, om2 = om * om;
  const R wsm = c.wss * (om2 * om2);
  R Zf = 0;
  if (fs > R(0)) Zf = wsm / (R(0.4) * (Uf + 2 * wsm));
  const R src = S.ketdinh ? source_chs(c, wsm, Zf, fs, fw, vth, Hm)
                          : source_nchs(c, wsm, Zf, Uf, R(1) / Hm, fs);
  S.dH[pos] += double(c.dT / (1 - c.Dorong) * (src + tH));
}

// The bed feedback (HydistOptions::bed_feedback; the reference computes dH
// but never applies it): dH > 0 deepens the bed (dH = dT/(1-porosity)
// (source + divergence), sediment_transport.cpp:535), so htaiz = htaiz0 + dH
// at z points, a wet node's depth h is its initial depth plus the mean dH
// of the four cells around it (a node at NANGDAY or below stays), and Kx1,
// Ky1 follow from the new depths as Onetime_init computes them
// (support_funcs.cpp:63-67). Thread (i, j) writes node (i, j) for i <= N+1,
// j <= M+1 and the z point (i, j) for 1 <= i <= N, 1 <= j <= M, computing
// the neighbouring nodes it needs from h0 and dH itself (nothing it reads
// is written by another thread).
template <class R, int BATCH = 0>
__global__ void k_bed_feedback(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (i > S.N + 1 || j > S.M + 1) return;
  const int W = S.W, p = i * W + j;
  const double* dH = S.dH;
  const double ND = c.NANGDAY;
  auto node = [&](int q) {
    const double b0 = S.h0[q];
    return b0 > ND ? b0 + 0.25 * (dH[q] + dH[q + W] + dH[q + 1] + dH[q + W + 1]) : b0;
  };
  const double hp = node(p);
  double* h = const_cast<double*>(S.h);
  h[p] = hp;
  if (i < 1 || j < 1 || i > S.N || j > S.M) return;
  const double hl = node(p - 1), hu = node(p - W);
  const_cast<double*>(S.htaiz)[p] = S.htaiz0[p] + dH[p];
  const double g = c.g, e = -2 * (double)c.mu_mn;
  if (hl + hp != 0)
    const_cast<R*>(S.Kx1)[p] =
        (R)(g * pow((hl + hp) * 0.5, e) * pow((S.hsnham[p - 1] + S.hsnham[p]) * 0.5, 2.0));
  if (hu + hp != 0)
    const_cast<R*>(S.Ky1)[p] =
        (R)(g * pow((hu + hp) * 0.5, e) * pow((S.hsnham[p - W] + S.hsnham[p]) * 0.5, 2.0));
}

template <class R>
void launch_bed_feedback(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st,
                         const Batch<R>& b) {
  const dim3 g(cdiv(S.M + 2, 128), S.N + 2, grid_z(b));
  if (b.n > 0) k_bed_feedback<R, 1><<<g, 128, 0, st>>>(S, c, b);
  else k_bed_feedback<R, 0><<<g, 128, 0, st>>>(S, c, b);
}
template void launch_bed_feedback<double>(const StateT<double>&, const CoefT<double>&, cudaStream_t,
                                          const Batch<double>&);
template void launch_bed_feedback<float>(const StateT<float>&, const CoefT<float>&, cudaStream_t,
                                         const Batch<float>&);

// The rows of a concentration sweep (_FSj / _FSi_calculate__mactrix_coeff,
// sediment_transport.cpp:204-313, 51-164, without the segment-end
// conditions, which the sweep applies) of every cell of rows 2..N, columns
// 2..M into the first four arrays of StateT::pre (A, B, C, D), ahead of the
// sweep: one thread per cell, adjacent threads on adjacent cells. DIR 0:
// the i-sweep (along i, the cell before is (i-1, j)), 1: the j-sweep.
template <class R, int DIR, int BATCH = 0>
__device__ __forceinline__ void fs_rows_cells(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int i = blockIdx.y + 2;
  if (i > S.N || j > S.M) return;
  const int W = S.W, g = i * W + j, gp = DIR == 0 ? g - W : g - 1;
  const R* vel = DIR == 0 ? S.tu : S.tv;
  const R hk_c = DIR == 0 ? S.Htdu[g] * S.Kx[g] : S.Htdv[g] * S.Ky[g];
  const R hk_p = DIR == 0 ? S.Htdu[gp] * S.Kx[gp] : S.Htdv[gp] * S.Ky[gp];
  R A, B, C, D;
  fs_cell(S, c, DIR == 0, i, j, vel[g], hk_c, vel[gp], hk_p, S.clock[0], S.src_start, A, B, C, D);
  const size_t n = (size_t)W * S.H;
  R* q = S.pre + g;
  q[0] = A;
  q[n] = B;
  q[2 * n] = C;
  q[3 * n] = D;
}

constexpr int FS_ROWS = 8;

template <class R, int BATCH = 0>
__global__ void k_update_fs(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  const StateT<R> S = member_state<BATCH>(S_arg, b_arg);
  const CoefT<R> c = member_coef<BATCH>(c_arg, b_arg);
  // FS = tFS on rows 1..N, columns 1..M; FS_ROWS rows per thread, every
  // load before the first store
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i0 = blockIdx.y * FS_ROWS + 1;
  if (j > S.M) return;
  R v[FS_ROWS];
#pragma unroll
  for (int r = 0; r < FS_ROWS; ++r) v[r] = i0 + r <= S.N ? S.tFS[(i0 + r) * S.W + j] : R(0);
#pragma unroll
  for (int r = 0; r < FS_ROWS; ++r)
    if (i0 + r <= S.N) S.FS[(i0 + r) * S.W + j] = v[r];
  bool fin = true;
#pragma unroll
  for (int r = 0; r < FS_ROWS; ++r) fin &= (bool)isfinite(v[r]);
  if (!fin) atomicOr(S.err, DEV_NONFINITE);
}

// Entry points of the passes above: the single-scenario kernels unbounded,
// the batch ones (suffix _b) under HYD_CELL_BOUNDS. A bound changes ptxas's
// register choice even where it does not bind, so the two are separate
// kernels.
// (the single-scenario ones bounded as well where that measured faster: in FP64
// the bed load at seven CTAs per SM and the concentration rows at ten, 7 us
// less per step on 2048x1024; in FP32 the bounds keep ptxas's own choice,
// 48 and 32 registers, a looser bound having cost 4 us)
template <class R, int BATCH = 0>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 7 : 10)
    k_bed_load(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  bed_load_cells<R, BATCH>(S_arg, c_arg, b_arg);
}
template <class R>
__global__ void HYD_CELL_BOUNDS k_bed_load_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  bed_load_cells<R, 1>(S_arg, c_arg, b_arg);
}

template <class R, int DIR, int BATCH = 0>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 10 : 16)
    k_fs_rows(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  fs_rows_cells<R, DIR, BATCH>(S_arg, c_arg, b_arg);
}
template <class R, int DIR>
__global__ void HYD_CELL_BOUNDS k_fs_rows_b(StateT<R> S_arg, CoefT<R> c_arg, Batch<R> b_arg) {
  fs_rows_cells<R, DIR, 1>(S_arg, c_arg, b_arg);
}

template <class R>
void launch_sediment(const StateT<R>& S, const CoefT<R>& c, bool xdir, bool bed, cudaStream_t st,
                     Trace* tr, const Batch<R>& b) {
  // Find_VTH + hesoK ran in the half-step's commit (k_commit_a/k_commit_b)
  if (tr) tr->kbegin(st, xdir ? KS_FS_X : KS_FS_Y);
  const unsigned z = grid_z(b);
  {
    const dim3 gr(cdiv(S.M - 1, 128), S.N - 1, z);
    if (b.n > 0) {
      if (xdir) k_fs_rows_b<R, 0><<<gr, 128, 0, st>>>(S, c, b);
      else k_fs_rows_b<R, 1><<<gr, 128, 0, st>>>(S, c, b);
    } else {
      if (xdir) k_fs_rows<R, 0, 0><<<gr, 128, 0, st>>>(S, c, b);
      else k_fs_rows<R, 1, 0><<<gr, 128, 0, st>>>(S, c, b);
    }
  }
  const int nfs = 1 + launch_fs_sweep(S, c, xdir ? 0 : 1, st, b);
  if (tr) tr->kend(st, xdir ? KS_FS_X : KS_FS_Y);
  const dim3 gfs(cdiv(S.M, 128), cdiv(S.N, FS_ROWS), z);
  if (b.n > 0) k_update_fs<R, 1><<<gfs, 128, 0, st>>>(S, c, b);
  else k_update_fs<R, 0><<<gfs, 128, 0, st>>>(S, c, b);
  int launched = nfs + 1;
  if (bed && S.N >= 5) {
    // the bed change once per step, after the j-sweep (engine.cpp:290-293)
    // the flux Qb was computed by this step's second commit (k_commit_b)
    const dim3 gl(cdiv(S.M - 1, 128), S.N - 4, z);
    if (b.n > 0) k_bed_load_b<R><<<gl, 128, 0, st>>>(S, c, b);
    else k_bed_load<R, 0><<<gl, 128, 0, st>>>(S, c, b);
    launched += 1;
    if (S.bed_fb) {
      launch_bed_feedback(S, c, st, b);
      ++launched;
    }
  }
  if (tr) tr->mark(st, xdir ? PH_SEDIMENT_X : PH_SEDIMENT_Y, launched);
}

template void launch_sediment<double>(const StateT<double>&, const CoefT<double>&, bool, bool,
                                      cudaStream_t, Trace*, const Batch<double>&);
template void launch_sediment<float>(const StateT<float>&, const CoefT<float>&, bool, bool,
                                     cudaStream_t, Trace*, const Batch<float>&);

}  // namespace hyd
