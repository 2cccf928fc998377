// sediment.cu -- suspended-sediment concentration step on the GPU.
//
// Kernels (reference kernel each one replaces in brackets):
//   k_vth_heso     [Find_VTH + hesoK, sediment_transport.cpp:575-602, 539-573]
//   the sweeps     [Scan_FSj/Scan_FSi + tridiagSolver + FSj/FSi_extract_
//                   solution, :51-349, 604-651]: the partitioned line solver
//                   with FSGen (sweep.cu), cell rows in sediment_cell.cuh
//   k_update_fs    [Update_FS, :654-663]
#include "common.cuh"
#include "hydro.cuh"
#include "sediment_cell.cuh"

namespace hyd {

// Find_VTH (rows/columns 2..) and hesoK (1..) over one grid: both read the
// committed velocities of the same cells.
__global__ void k_vth_heso(State S, Coef c, int i_hi) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i = blockIdx.y + 1;
  if (i > i_hi || j > S.M) return;
  const int W = S.W, p = i * W + j;
  const double tu = S.tu[p], tv = S.tv[p];
  if (i >= 2 && j >= 2) {
    if ((S.htaiz[p] > c.NANGDAY) && (S.Hmoi[p] > c.H_TINH)) {
      const double ut = (tu + S.tu[p - W]) * 0.5;
      const double vt = (tv + S.tv[p - 1]) * 0.5;
      S.VTH[p] = sqrt(ut * ut + vt * vt);
    } else {
      S.VTH[p] = 0;
    }
  }
  const double hp = S.h[p];
  const double Hu = S.Htdu[p], Hv = S.Htdv[p];
  if (Hu > 0) {
    const double Cz = 18 * log(12 * Hu / c.Ks);
    const double k = 5.93 * c.sqrt_g * (S.h[p - 1] + hp) * 0.25 * fabs(tu) / Cz;
    S.Kx[p] = fmin(100.0, fmax(5.0, k));
  }
  if (Hv > 0) {
    const double Cz = 18 * log(12 * Hv / c.Ks);
    const double k = 5.93 * c.sqrt_g * (S.h[p - W] + hp) * 0.25 * fabs(tv) / Cz;
    S.Ky[p] = fmin(100.0, fmax(5.0, k));
  }
}

__global__ void k_update_fs(State S) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i = blockIdx.y + 1;
  if (i > S.N || j > S.M) return;
  const int g = i * S.W + j;
  S.FS[g] = S.tFS[g];
}

void launch_sediment(const State& S, const Coef& c, double s_start, bool xdir, cudaStream_t st,
                     Trace* tr) {
  // first half: Find_VTH/hesoK over rows to N; second half: to N-1
  // (launch shape of engine.cpp:259-260 never reaches row N)
  const int i_hi = xdir ? S.N : S.N - 1;
  k_vth_heso<<<dim3(cdiv(S.M, 128), i_hi), 128, 0, st>>>(S, c, i_hi);
  if (tr) tr->kbegin(st, xdir ? KS_FS_X : KS_FS_Y);
  launch_fs_sweep(S, c, xdir ? 0 : 1, s_start, st);
  if (tr) tr->kend(st, xdir ? KS_FS_X : KS_FS_Y);
  k_update_fs<<<dim3(cdiv(S.M, 128), S.N), 128, 0, st>>>(S);
  if (tr) tr->mark(st, xdir ? PH_SEDIMENT_X : PH_SEDIMENT_Y, 3);
}

}  // namespace hyd
