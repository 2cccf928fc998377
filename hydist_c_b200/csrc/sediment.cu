// sediment.cu -- suspended-sediment concentration sweeps on the GPU.
//
// Kernels (reference kernel each one replaces in brackets):
//   k_find_vth     [Find_VTH, sediment_transport.cpp:575-602]
//   k_heso_k       [hesoK, :539-573]
//   k_fs_sweep_x   [Scan_FSj + tridiagSolver + FSj_extract_solution,
//                   :204-349, 628-651; engine.cpp:150-170] one thread per column
//   k_fs_sweep_y   [Scan_FSi + tridiagSolver + FSi_extract_solution,
//                   :51-201, 604-625; engine.cpp:259-282] one thread per row
//   k_update_fs    [Update_FS, :654-663]
#include "common.cuh"
#include "hydro.cuh"

namespace hyd {

__global__ void k_find_vth(State S, Coef c, int i_hi) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int i = blockIdx.y + 2;
  if (i > i_hi || j > S.M) return;
  const int W = S.W, p = i * W + j;
  if ((S.htaiz[p] > c.NANGDAY) && (S.Hmoi[p] > c.H_TINH)) {
    const double ut = (S.tu[p] + S.tu[p - W]) * 0.5;
    const double vt = (S.tv[p] + S.tv[p - 1]) * 0.5;
    S.VTH[p] = sqrt(ut * ut + vt * vt);
  } else {
    S.VTH[p] = 0;
  }
}

__global__ void k_heso_k(State S, Coef c, int i_hi) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i = blockIdx.y + 1;
  if (i > i_hi || j > S.M) return;
  const int W = S.W, p = i * W + j;
  const double sg = sqrt(c.g);
  if (S.Htdu[p] > 0) {
    const double Cz = 18 * log(12 * S.Htdu[p] / c.Ks);
    const double k = 5.93 * sg * (S.h[p - 1] + S.h[p]) * 0.25 * fabs(S.tu[p]) / Cz;
    S.Kx[p] = fmin(100.0, fmax(5.0, k));
  }
  if (S.Htdv[p] > 0) {
    const double Cz = 18 * log(12 * S.Htdv[p] / c.Ks);
    const double k = 5.93 * sg * (S.h[p - W] + S.h[p]) * 0.25 * fabs(S.tv[p]) / Cz;
    S.Ky[p] = fmin(100.0, fmax(5.0, k));
  }
}

// source_chs (sediment_transport.cpp:11-38)
__device__ __forceinline__ double source_chs(const Coef& c, double wsm, double Zf, double fs,
                                             double fw, double vth, double h_moi) {
  double toee = c.Toe;
  const double todd = c.Tod;
  double S = 0;
  const double tob = c.ro * fw * (vth * vth);
  if (h_moi > c.ghtoe) toee = toee * (1 + c.hstoe * ((h_moi - c.ghtoe)));
  if (tob > toee) {
    S = c.Mbochat / c.ros * (tob - toee) / toee;
  } else if (tob < todd) {
    const double Pd = 1 - (tob / todd);
    const double beta = 1 + (Zf / (1.25 + 4.75 * pow(Pd, 2.5)));
    const double Cb = beta * fs;
    S = -wsm * Cb * Pd;
  }
  return S;
}

// source_nchs (sediment_transport.cpp:41-49)
__device__ __forceinline__ double source_nchs(const Coef& c, double wsm, double Zf, double Uf,
                                              double h_moi, double fs) {
  const double gamac = 0.434 + 5.975 * Zf + 2.888 * Zf * Zf;
  const double Tx = fmax(0.0, (Uf * Uf - c.Ufr * c.Ufr) / (c.Ufr * c.Ufr));
  const double Cac = 0.015 * c.dm * pow(Tx, 1.5) * pow(c.Dxr, (-0.3)) / (0.05 * h_moi);
  return wsm * (Cac - gamac * fs);
}

// One cell's row of a concentration sweep: xdir = _FSj (:204-313), else
// _FSi (:51-164).
__device__ __forceinline__ void fs_cell(const State& S, const Coef& c, bool xdir, int i, int j,
                                        double tt, double s_start, double& A, double& B,
                                        double& Cc, double& D) {
  const int w = S.W, pos = i * w + j;
  const double* Hm = S.Hmoi;
  const double* FS = S.FS;
  const double dX = c.dX, dY = c.dY, dT = c.dT, H_TINH = c.H_TINH;
  const double cc = 18 * log(12 * Hm[pos] / c.Ks);
  const double Uf = sqrt(c.g) * fabs(S.VTH[pos]) / cc;
  const double wsm = c.wss * pow((1 - FS[pos]), 4.0);
  double Zf = 0, Sx;
  double gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
  if (FS[pos] > 0.00001) Zf = wsm / (0.4 * (Uf + 2 * wsm));
  if (S.ketdinh)
    Sx = source_chs(c, wsm, Zf, FS[pos], S.Fw[pos], S.VTH[pos], Hm[pos]);
  else
    Sx = source_nchs(c, wsm, Zf, Uf, Hm[pos], FS[pos]);
  if (tt < s_start) Sx = 0;
  double p = 0, q = 0;
  if (xdir) {
    A = -gamav * 0.5 * (S.tu[pos] + S.tu[pos - w]) / (dX * 2) -
        S.Htdu[pos - w] * S.Kx[pos - w] / (Hm[pos] * (dX * dX));
    Cc = gamav * 0.5 * (S.tu[pos] + S.tu[pos - w]) / (dX * 2) -
         S.Htdu[pos] * S.Kx[pos] / (Hm[pos] * (dX * dX));
    B = 2.0 / dT + (S.Htdu[pos] * S.Kx[pos] + S.Htdu[pos - w] * S.Kx[pos - w]) / (Hm[pos] * (dX * dX));
    if ((Hm[pos - 1] > H_TINH) && (Hm[pos + 2] > H_TINH)) p = (FS[pos + 1] - FS[pos]);
    if ((Hm[pos - 2] > H_TINH) && (Hm[pos + 1] > H_TINH)) q = (FS[pos] - FS[pos - 1]);
    p = (1 / (Hm[pos] * (dY * dY))) * (S.Htdv[pos] * S.Ky[pos] * p - S.Htdv[pos - 1] * S.Ky[pos - 1] * q);
    if ((Hm[pos - 2] > H_TINH) && (Hm[pos + 2] > H_TINH)) {
      q = (FS[pos + 1] - FS[pos - 1]) / (dY * 2);
      q = (S.tv[pos] + S.tv[pos - 1]) * 0.5 * q * gamav;
    } else {
      q = 0;
    }
  } else {
    gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
    A = -gamav * 0.5 * (S.tv[pos - 1] + S.tv[pos]) / (dY * 2) -
        S.Htdv[pos - 1] * S.Ky[pos - 1] / (Hm[pos] * (dY * dY));
    Cc = gamav * 0.5 * (S.tv[pos - 1] + S.tv[pos]) / (dY * 2) -
         S.Htdv[pos] * S.Ky[pos] / (Hm[pos] * (dY * dY));
    B = 2.0 / dT + (S.Htdv[pos] * S.Ky[pos] + S.Htdv[pos - 1] * S.Ky[pos - 1]) / (Hm[pos] * (dY * dY));
    if ((Hm[pos + 2 * w] > H_TINH) && (Hm[pos - w] > H_TINH)) p = (FS[pos + w] - FS[pos]);
    if (Hm[pos - 2 * w] > H_TINH && Hm[pos + w] > H_TINH) q = (FS[pos] - FS[pos - w]);
    p = (1 / (Hm[pos] * (dX * dX))) * (S.Htdu[pos] * S.Kx[pos] * p - S.Htdu[pos - w] * S.Kx[pos - w] * q);
    if (Hm[pos + 2 * w] > H_TINH && Hm[pos - 2 * w] > H_TINH) {
      q = (FS[pos + w] - FS[pos - w]) / (dX * 2);
      q = (S.tu[pos] + S.tu[pos - w]) * 0.5 * q * gamav;
    } else {
      q = 0;
    }
  }
  D = FS[pos] / (dT * 0.5) - q + p + (Sx / Hm[pos]);
}

// Column i-sweep of the concentration (first half-step).
__global__ void __launch_bounds__(128) k_fs_sweep_x(State S, Coef c, double tt, double s_start) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 3;
  if (j > S.M - 1) return;
  const int w = S.W, N = S.N;
  double* Ap = S.Ap + j;
  double* Bp = S.Bp + j;
  const int ld = S.ld;
  for (int k = 0; k < S.mocj[j]; ++k) {
    const int first = S.dauj[j * SEG + k], last = S.cuoij[j * SEG + k];
    if (last < first + 2) continue;
    const bool br1 = (first > 2) || ((first == 2) && ((S.h[1 * w + j] + S.h[1 * w + j - 1]) * 0.5 == c.NANGDAY));
    const bool br2 = (last < N) || ((last == N) && ((S.h[N * w + j] + S.h[N * w + j - 1]) * 0.5 == c.NANGDAY));
    const int sn = last - first - 2;
    double ap = 0, bp = 0, xs = 0;
    for (int i = first + 1; i <= last - 1; ++i) {
      double A, B, Cc, D;
      fs_cell(S, c, true, i, j, tt, s_start, A, B, Cc, D);
      if (i == first + 1) {
        if ((br1) || (S.tu[first * w + j] == 0)) B += A;
        else D -= A * S.FS[first * w + j];
      }
      if (i == last - 1) {
        if ((br2) && (S.tu[last * w + j] == 0)) B += Cc;
        else D -= Cc * S.FS[last * w + j];
      }
      const int kk = i - (first + 1);
      if (kk == 0) {
        if (sn == 0) {
          xs = D / B;
          continue;
        }
        ap = -Cc / B;
        bp = D / B;
      } else if (kk < sn) {
        const double ep = A * ap + B;
        ap = -Cc / ep;
        bp = (D - (A * bp)) / ep;
      } else {
        xs = (D - (A * bp)) / (B + (A * ap));
        continue;
      }
      Ap[(size_t)i * ld] = ap;
      Bp[(size_t)i * ld] = bp;
    }
    // back substitution + FSj_extract_solution (:316-349)
    double xr = xs;
    for (int i = last - 1; i >= first + 1; --i) {
      double x = xr;
      if (i < last - 1) x = Bp[(size_t)i * ld] + Ap[(size_t)i * ld] * xr;
      xr = x;
      const int p = i * w + j;
      const double tf = (x < 0) ? c.NDnen : x;
      S.tFS[p] = tf;
      if (i == last - 1)
        S.tFS[last * w + j] = ((br2) || (S.tu[p + w] == 0)) ? tf : S.FS[last * w + j];
      if (i == first + 1)
        S.tFS[first * w + j] = ((br1) || (S.tu[p - w] == 0)) ? tf : S.FS[first * w + j];
    }
  }
}

// Row j-sweep of the concentration (second half-step).
__global__ void __launch_bounds__(128) k_fs_sweep_y(State S, Coef c, double tt, double s_start) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 3;
  if (i > S.N - 1) return;
  const int w = S.W, M = S.M;
  double* Ap = S.Ap + i;
  double* Bp = S.Bp + i;
  const int ld = S.ld;
  for (int k = 0; k < S.moci[i]; ++k) {
    const int first = S.daui[i * SEG + k], last = S.cuoii[i * SEG + k];
    if (last < first + 2) continue;
    const bool br1 = (first > 2) || ((first == 2) && ((S.h[i * w + first - 1] + S.h[(i - 1) * w + first - 1]) * 0.5 == c.NANGDAY));
    const bool br2 = (last < M) || ((last == M) && ((S.h[i * w + last] + S.h[(i - 1) * w + last]) * 0.5 == c.NANGDAY));
    const int sn = last - first - 2;
    double ap = 0, bp = 0, xs = 0;
    for (int j = first + 1; j <= last - 1; ++j) {
      double A, B, Cc, D;
      fs_cell(S, c, false, i, j, tt, s_start, A, B, Cc, D);
      if (j == first + 1) {
        if ((br1) || (S.tv[i * w + first] == 0)) B = B + A;
        else D = D - A * S.FS[i * w + first];
      }
      if (j == last - 1) {
        if ((br2) || (S.tv[i * w + last] == 0)) B = B + Cc;
        else D = D - Cc * S.FS[i * w + last];
      }
      const int kk = j - (first + 1);
      if (kk == 0) {
        if (sn == 0) {
          xs = D / B;
          continue;
        }
        ap = -Cc / B;
        bp = D / B;
      } else if (kk < sn) {
        const double ep = A * ap + B;
        ap = -Cc / ep;
        bp = (D - (A * bp)) / ep;
      } else {
        xs = (D - (A * bp)) / (B + (A * ap));
        continue;
      }
      Ap[(size_t)j * ld] = ap;
      Bp[(size_t)j * ld] = bp;
    }
    double xr = xs;
    for (int j = last - 1; j >= first + 1; --j) {
      double x = xr;
      if (j < last - 1) x = Bp[(size_t)j * ld] + Ap[(size_t)j * ld] * xr;
      xr = x;
      const int p = i * w + j;
      const double tf = (x < 0) ? c.NDnen : x;
      S.tFS[p] = tf;
      if (j == last - 1)
        S.tFS[i * w + last] = ((br2) || (S.tv[i * w + last] == 0)) ? tf : S.FS[i * w + last];
      if (j == first + 1)
        S.tFS[i * w + first] = ((br1) || (S.tv[i * w + first] == 0)) ? tf : S.FS[i * w + first];
    }
  }
}

__global__ void k_update_fs(State S) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i = blockIdx.y + 1;
  if (i > S.N || j > S.M) return;
  const int g = i * S.W + j;
  S.FS[g] = S.tFS[g];
}

void launch_sediment(const State& S, const Coef& c, double t, double s_start, bool xdir,
                     cudaStream_t st, Trace* tr) {
  // first half: Find_VTH/hesoK over rows to N; second half: to N-1
  // (launch shape of engine.cpp:259-260 never reaches row N)
  const int i_hi = xdir ? S.N : S.N - 1;
  k_find_vth<<<dim3(cdiv(S.M - 1, 128), i_hi - 1), 128, 0, st>>>(S, c, i_hi);
  k_heso_k<<<dim3(cdiv(S.M, 128), i_hi), 128, 0, st>>>(S, c, i_hi);
  if (xdir)
    k_fs_sweep_x<<<cdiv(S.M - 3, 128), 128, 0, st>>>(S, c, t, s_start);
  else
    k_fs_sweep_y<<<cdiv(S.N - 3, 128), 128, 0, st>>>(S, c, t, s_start);
  k_update_fs<<<dim3(cdiv(S.M, 128), S.N), 128, 0, st>>>(S);
  if (tr) tr->mark(st, xdir ? PH_SEDIMENT_X : PH_SEDIMENT_Y, 4);
}

}  // namespace hyd
