/*
 * hydist_gtsv_device.cuh -- the reference's device-side tridiagonal solve
 * gtsv_spike_partial_diag_pivot_v1 (gtsv.h:7, gtsv.cpp:88-193) with its
 * signature, header-only, for device code written against the reference.
 *
 * Replaces: __device__ void gtsv_spike_partial_diag_pivot_v1(const double* dl,
 *   const double* d, const double* du, double* b, double* x, const int m)
 * (gtsv.h:7). The reference's version launches a SPIKE solver with diagonal
 * pivoting per tile as child grids from the calling thread (dynamic
 * parallelism, cudaMalloc'd buffers, never synchronised before return);
 * this one solves the system in the calling thread, sequentially, by
 * Gaussian elimination with the same kind of pivoting, and x holds the
 * solution when it returns.
 *
 * System: m rows; row i is dl[i] x[i-1] + d[i] x[i] + du[i] x[i+1] = b[i]
 * (dl[0] and du[m-1] are not read). b is only read. Pivoting: at each step
 * either the current diagonal (1x1 pivot) or the 2x2 block of the current
 * and the next row is eliminated, chosen by the Bunch-Kaufman criterion with
 * kappa = (sqrt(5)-1)/2: the 1x1 pivot d' is taken when
 * |d'| sigma >= kappa |du[k] dl[k+1]|, sigma the largest magnitude among the
 * entries coupling the next two rows (Bunch and Kaufman, Math. Comp. 31,
 * 1977; its tridiagonal form is the one of Erway and Marcia and of Chang et
 * al., SC'12, which the reference's per-tile solver follows).
 *
 * Memory: the modified pivots come from the device heap (malloc, m doubles
 * and m/8 bytes), as the reference's device-side cudaMalloc does; raise
 * cudaLimitMallocHeapSize for many concurrent large solves. If the heap is
 * exhausted x is filled with NaN. For batches of systems from the host use
 * hydist_gtsv_batched (hydist_capi.h) instead.
 *
 * A translation unit must not include both this header and the reference's
 * gtsv.h: they define the same function.
 */
#ifndef HYDIST_GTSV_DEVICE_CUH
#define HYDIST_GTSV_DEVICE_CUH

#include <cuda_runtime.h>

__device__ inline void gtsv_spike_partial_diag_pivot_v1(const double* dl, const double* d,
                                                        const double* du, double* b, double* x,
                                                        const int m) {
  if (m <= 0) return;
  const double kappa = 0.6180339887498949;  // (sqrt(5) - 1) / 2
  // per row: the modified pivot (1x1), or for a 2x2 block its first row's
  // modified diagonal and its second row's determinant; bit i of `two` marks
  // the second row of a 2x2 block. x holds the modified right-hand side.
  double* piv = static_cast<double*>(malloc(sizeof(double) * (size_t)m + (size_t)(m + 7) / 8));
  if (!piv) {
    for (int i = 0; i < m; ++i) x[i] = __longlong_as_double(0x7ff8000000000000LL);
    return;
  }
  unsigned char* two = reinterpret_cast<unsigned char*>(piv + m);
  for (int i = 0; i < (m + 7) / 8; ++i) two[i] = 0;
  // forward elimination
  double dk = d[0], rk = b[0];
  int k = 0;
  while (k < m) {
    if (k == m - 1) {
      piv[k] = dk;
      x[k] = rk;
      break;
    }
    double sigma = fmax(fmax(fabs(du[k]), fabs(dl[k + 1])), fabs(d[k + 1]));
    if (k + 2 < m) sigma = fmax(sigma, fmax(fabs(du[k + 1]), fabs(dl[k + 2])));
    if (fabs(dk) * sigma >= kappa * fabs(du[k] * dl[k + 1])) {
      // 1x1 pivot: row k+1 loses its entry in column k
      piv[k] = dk;
      x[k] = rk;
      const double l = dl[k + 1] / dk;
      dk = d[k + 1] - l * du[k];
      rk = b[k + 1] - l * rk;
      k += 1;
    } else {
      // 2x2 pivot [[dk, du[k]], [dl[k+1], d[k+1]]]: row k+2 loses its entry
      // in column k+1
      const double det = dk * d[k + 1] - du[k] * dl[k + 1];
      piv[k] = dk;
      piv[k + 1] = det;
      two[(k + 1) >> 3] |= (unsigned char)(1u << ((k + 1) & 7));
      x[k] = rk;
      x[k + 1] = b[k + 1];
      if (k + 2 < m) {
        // row k+2 minus dl[k+2] times row 2 of the block's inverse applied to
        // the block's rows: (B^-1)_{22} = dk / det
        const double l = dl[k + 2] / det;
        rk = b[k + 2] - l * (dk * b[k + 1] - dl[k + 1] * rk);
        dk = d[k + 2] - l * dk * du[k + 1];
      }
      k += 2;
    }
  }
  // back substitution
  double xn = 0.0;  // x[i+1]
  int i = m - 1;
  while (i >= 0) {
    if (two[i >> 3] & (1u << (i & 7))) {
      // rows i-1, i: [[p, du[i-1]], [dl[i], d[i]]] [x_{i-1}; x_i] = [r0; r1]
      const double p = piv[i - 1], det = piv[i];
      const double r0 = x[i - 1];
      const double r1 = x[i] - (i + 1 < m ? du[i] * xn : 0.0);
      const double xi = (p * r1 - dl[i] * r0) / det;
      const double xi1 = (d[i] * r0 - du[i - 1] * r1) / det;
      x[i] = xi;
      x[i - 1] = xi1;
      xn = xi1;
      i -= 2;
    } else {
      const double xi = (x[i] - (i + 1 < m ? du[i] * xn : 0.0)) / piv[i];
      x[i] = xi;
      xn = xi;
      i -= 1;
    }
  }
  free(piv);
}

#endif
