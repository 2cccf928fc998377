// gtsv_device_check.cu -- TEST PROGRAM for include/hydist_gtsv_device.cuh.
//
// Solves seeded tridiagonal systems with gtsv_spike_partial_diag_pivot_v1,
// one system per thread, and prints, per kind of system, the largest
// residual |A x - b|_inf / (|A|_inf |x|_inf + |b|_inf) over the batch:
//   dominant  diagonally dominant (b = |a|+|c|+U(0.1,1)), as the sweeps make;
//   zerodiag  diagonal U(-1,1) with every third diagonal entry zero, which
//             needs 2x2 pivots (Thomas without pivoting divides by zero);
//   small     lengths 1 and 2.
// usage: gtsv_device_check  (prints "kind maxres" lines; exit 0)
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/hydist_gtsv_device.cuh"

__global__ void solve_all(const double* dl, const double* d, const double* du, double* b,
                          double* x, const int* off, const int* len, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int o = off[s];
  gtsv_spike_partial_diag_pivot_v1(dl + o, d + o, du + o, b + o, x + o, len[s]);
}

static unsigned long long rng = 20261203ull;
static double uni() {  // U(0,1), splitmix64
  rng += 0x9E3779B97F4A7C15ull;
  unsigned long long z = rng;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (z >> 11) * (1.0 / 9007199254740992.0);
}

static int check(const char* kind, int nsys, int minlen, int maxlen, bool zerodiag) {
  std::vector<int> off(nsys), len(nsys);
  int n = 0;
  for (int s = 0; s < nsys; ++s) {
    off[s] = n;
    len[s] = minlen + (int)(uni() * (maxlen - minlen + 1));
    if (len[s] > maxlen) len[s] = maxlen;
    n += len[s];
  }
  std::vector<double> dl(n), d(n), du(n), b(n), x(n);
  for (int i = 0; i < n; ++i) {
    dl[i] = 2 * uni() - 1;
    du[i] = 2 * uni() - 1;
    if (zerodiag) d[i] = (i % 3 == 0) ? 0.0 : 2 * uni() - 1;
    else d[i] = std::fabs(dl[i]) + std::fabs(du[i]) + 0.1 + 0.9 * uni();
    b[i] = 2 * uni() - 1;
  }
  double *gdl, *gd, *gdu, *gb, *gx;
  int *goff, *glen;
  cudaMalloc(&gdl, n * 8);
  cudaMalloc(&gd, n * 8);
  cudaMalloc(&gdu, n * 8);
  cudaMalloc(&gb, n * 8);
  cudaMalloc(&gx, n * 8);
  cudaMalloc(&goff, nsys * 4);
  cudaMalloc(&glen, nsys * 4);
  cudaMemcpy(gdl, dl.data(), n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(gd, d.data(), n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(gdu, du.data(), n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(gb, b.data(), n * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(goff, off.data(), nsys * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(glen, len.data(), nsys * 4, cudaMemcpyHostToDevice);
  solve_all<<<(nsys + 127) / 128, 128>>>(gdl, gd, gdu, gb, gx, goff, glen, nsys);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    printf("error %s\n", cudaGetErrorString(e));
    return 1;
  }
  cudaMemcpy(x.data(), gx, n * 8, cudaMemcpyDeviceToHost);
  std::vector<double> b2(n);
  cudaMemcpy(b2.data(), gb, n * 8, cudaMemcpyDeviceToHost);
  double worst = 0;
  for (int s = 0; s < nsys; ++s) {
    const int o = off[s], m = len[s];
    double rmax = 0, amax = 0, xmax = 0, bmax = 0;
    for (int i = 0; i < m; ++i) {
      double r = d[o + i] * x[o + i] - b[o + i];
      double a = std::fabs(d[o + i]);
      if (i > 0) {
        r += dl[o + i] * x[o + i - 1];
        a += std::fabs(dl[o + i]);
      }
      if (i + 1 < m) {
        r += du[o + i] * x[o + i + 1];
        a += std::fabs(du[o + i]);
      }
      rmax = std::fmax(rmax, std::fabs(r));
      amax = std::fmax(amax, a);
      xmax = std::fmax(xmax, std::fabs(x[o + i]));
      bmax = std::fmax(bmax, std::fabs(b[o + i]));
    }
    const double res = rmax / (amax * xmax + bmax);
    if (!(res <= worst)) worst = std::isnan(res) ? INFINITY : std::fmax(worst, res);
  }
  bool b_kept = true;
  for (int i = 0; i < n; ++i) b_kept = b_kept && (b2[i] == b[i]);
  printf("%s %.3e b_unchanged=%d\n", kind, worst, b_kept ? 1 : 0);
  cudaFree(gdl);
  cudaFree(gd);
  cudaFree(gdu);
  cudaFree(gb);
  cudaFree(gx);
  cudaFree(goff);
  cudaFree(glen);
  return 0;
}

int main() {
  // one heap block of up to 1024 doubles per concurrent solve
  cudaDeviceSetLimit(cudaLimitMallocHeapSize, (size_t)64 << 20);
  int rc = 0;
  rc |= check("dominant", 2048, 16, 1024, false);
  rc |= check("zerodiag", 2048, 16, 1024, true);
  rc |= check("small", 256, 1, 2, false);
  return rc;
}
