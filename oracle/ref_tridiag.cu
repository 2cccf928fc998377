// ref_tridiag.cu -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's device Thomas solver, tridiag()
// (UVZSolver_multithread.cpp:19-43, compiled from the reference sources),
// one thread per system over a packed batch, and times it with CUDA events.
// This is the reference's own tridiagonal solver on the GPU; its launch
// wrapper tridiagSolver (:78-109) needs the mesh segment tables, so a plain
// per-system kernel stands in for it.
//
// usage: hydist_ref_tridiag <in.bin> <out.bin> [reps]
//   in.bin : int32 nsys, int32 total, int32 offsets[nsys], int32 lengths[nsys],
//            float64 dl[total], d[total], du[total], b[total]
//   out.bin: float64 x[total], then float64 mean_ms
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "UVZSolver_multithread.h"

static void ck(cudaError_t e, const char* w) {
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_tridiag: %s: %s\n", w, cudaGetErrorString(e));
    exit(3);
  }
}

__global__ void run_ref_tridiag(const int* off, const int* len, int nsys, double* dl, double* d,
                                double* du, double* b, double* x, double* Ap, double* Bp,
                                double* ep) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int o = off[s], n = len[s];
  if (n <= 0) return;
  tridiag(n - 1, dl + o, d + o, du + o, b + o, x + o, Ap + o, Bp + o, ep + o);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: hydist_ref_tridiag in.bin out.bin [reps]\n");
    return 2;
  }
  const int reps = argc > 3 ? atoi(argv[3]) : 10;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  int nsys = 0, total = 0;
  if (fread(&nsys, 4, 1, f) != 1 || fread(&total, 4, 1, f) != 1) return 2;
  std::vector<int> off(nsys), len(nsys);
  std::vector<double> a(4 * (size_t)total);
  if (fread(off.data(), 4, nsys, f) != (size_t)nsys || fread(len.data(), 4, nsys, f) != (size_t)nsys ||
      fread(a.data(), 8, a.size(), f) != a.size())
    return 2;
  fclose(f);
  for (int s = 0; s < nsys; ++s)
    if (off[s] < 0 || len[s] < 0 || (long)off[s] + len[s] > total) return 2;
  int *doff, *dlen;
  double *dbuf, *dx, *dAp, *dBp, *dep;
  ck(cudaMalloc(&doff, 4 * nsys), "malloc");
  ck(cudaMalloc(&dlen, 4 * nsys), "malloc");
  ck(cudaMalloc(&dbuf, 8 * a.size()), "malloc");
  ck(cudaMalloc(&dx, 8 * (size_t)total), "malloc");
  ck(cudaMalloc(&dAp, 8 * (size_t)total), "malloc");
  ck(cudaMalloc(&dBp, 8 * (size_t)total), "malloc");
  ck(cudaMalloc(&dep, 8 * (size_t)total), "malloc");
  ck(cudaMemcpy(doff, off.data(), 4 * nsys, cudaMemcpyHostToDevice), "h2d");
  ck(cudaMemcpy(dlen, len.data(), 4 * nsys, cudaMemcpyHostToDevice), "h2d");
  ck(cudaMemcpy(dbuf, a.data(), 8 * a.size(), cudaMemcpyHostToDevice), "h2d");
  double* dl = dbuf;
  double* d = dbuf + total;
  double* du = dbuf + 2 * (size_t)total;
  double* b = dbuf + 3 * (size_t)total;
  const int bs = 128, gs = (nsys + bs - 1) / bs;
  run_ref_tridiag<<<gs, bs>>>(doff, dlen, nsys, dl, d, du, b, dx, dAp, dBp, dep);
  ck(cudaDeviceSynchronize(), "warmup");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  for (int r = 0; r < reps; ++r)
    run_ref_tridiag<<<gs, bs>>>(doff, dlen, nsys, dl, d, du, b, dx, dAp, dBp, dep);
  cudaEventRecord(e1);
  ck(cudaEventSynchronize(e1), "run");
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  double mean = ms / reps;
  std::vector<double> x(total);
  ck(cudaMemcpy(x.data(), dx, 8 * (size_t)total, cudaMemcpyDeviceToHost), "d2h");
  f = fopen(argv[2], "wb");
  fwrite(x.data(), 8, total, f);
  fwrite(&mean, 8, 1, f);
  fclose(f);
  fprintf(stderr, "ref_tridiag: %d systems, %d unknowns, %.4f ms per batch\n", nsys, total, mean);
  return 0;
}
