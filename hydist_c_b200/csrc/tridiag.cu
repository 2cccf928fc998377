// tridiag.cu -- batched tridiagonal solver behind hydist_gtsv_batched.
//
// Replaces the reference's per-line solvers: tridiag()/tridiagSolver
// (UVZSolver_multithread.cpp:19-43, 78-109; serial Thomas, 32 redundant
// threads per line) and the SPIKE solver gtsv_spike_partial_diag_pivot_v1
// (gtsv.cpp:88-193, called per line with device-side allocation).
//
// Packed batch: system s occupies rows [off[s], off[s]+len[s]).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"

namespace hyd {

// Plain Thomas, one thread per system (the reference's algorithm; scratch
// for the forward sweep is the output array x and a second array w).
template <class T>
__global__ void k_thomas_batched(const T* __restrict__ dl, const T* __restrict__ d,
                                 const T* __restrict__ du, const T* __restrict__ b, T* __restrict__ x,
                                 T* __restrict__ w, const int* __restrict__ off,
                                 const int* __restrict__ len, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int o = off[s], n = len[s];
  if (n <= 0) return;
  const T* A = dl + o;
  const T* B = d + o;
  const T* C = du + o;
  const T* D = b + o;
  T* X = x + o;
  T* Wp = w + o;
  if (n == 1) {
    X[0] = D[0] / B[0];
    return;
  }
  T ap = -C[0] / B[0];
  T bp = D[0] / B[0];
  Wp[0] = ap;
  X[0] = bp;
  for (int i = 1; i < n - 1; ++i) {
    const T ep = A[i] * ap + B[i];
    ap = -C[i] / ep;
    bp = (D[i] - A[i] * bp) / ep;
    Wp[i] = ap;
    X[i] = bp;
  }
  T xr = (D[n - 1] - A[n - 1] * bp) / (B[n - 1] + A[n - 1] * ap);
  X[n - 1] = xr;
  for (int i = n - 2; i >= 0; --i) {
    xr = X[i] + Wp[i] * xr;
    X[i] = xr;
  }
}

}  // namespace hyd

namespace hyd {
void set_last_error(const char* m);
}

namespace {
struct Scratch {
  void* p = nullptr;
  size_t bytes = 0;
  int device = -1;
};
Scratch g_scratch;  // per process; guarded by the caller's stream order
}  // namespace

extern "C" int hydist_gtsv_batched(const void* dl, const void* d, const void* du, const void* b,
                                   void* x, const int32_t* offsets, const int32_t* lengths,
                                   int32_t nsys, int32_t dtype, int32_t algo, void* stream) {
  if (!dl || !d || !du || !b || !x || !offsets || !lengths || nsys < 0) return HYDIST_ERR_ARG;
  if (dtype != 0 && dtype != 1) return HYDIST_ERR_ARG;
  if (algo < 0 || algo > 3) return HYDIST_ERR_ARG;
  if (algo >= 2) {
    hyd::set_last_error("hydist_gtsv_batched: algo 2 and 3 are not implemented yet");
    return HYDIST_ERR_ARG;
  }
  if (nsys == 0) return HYDIST_OK;
  cudaStream_t st = (cudaStream_t)stream;
  // total rows = max(off+len): read the last system's extent from device
  // memory is avoided; the caller's x buffer bounds the rows, so scratch is
  // sized from the packed layout through a small reduction on the host side
  // of the caller. Here: scratch sized lazily to the x span.
  int last_off = 0, last_len = 0;
  if (cudaMemcpyAsync(&last_off, offsets + (nsys - 1), 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&last_len, lengths + (nsys - 1), 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return HYDIST_ERR_CUDA;
  const size_t rows = (size_t)last_off + (size_t)last_len;
  const size_t esz = dtype == 0 ? 8 : 4;
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_scratch.bytes < rows * esz || g_scratch.device != dev) {
    if (g_scratch.p) cudaFree(g_scratch.p);
    g_scratch.p = nullptr;
    g_scratch.bytes = 0;
    if (cudaMalloc(&g_scratch.p, rows * esz + 256) != cudaSuccess) return HYDIST_ERR_OOM;
    g_scratch.bytes = rows * esz;
    g_scratch.device = dev;
  }
  const int bs = 128, gs = (nsys + bs - 1) / bs;
  if (dtype == 0)
    hyd::k_thomas_batched<double><<<gs, bs, 0, st>>>(
        (const double*)dl, (const double*)d, (const double*)du, (const double*)b, (double*)x,
        (double*)g_scratch.p, offsets, lengths, nsys);
  else
    hyd::k_thomas_batched<float><<<gs, bs, 0, st>>>((const float*)dl, (const float*)d,
                                                    (const float*)du, (const float*)b, (float*)x,
                                                    (float*)g_scratch.p, offsets, lengths, nsys);
  if (cudaGetLastError() != cudaSuccess) return HYDIST_ERR_CUDA;
  return HYDIST_OK;
}

// ---- allocation-free variant --------------------------------------------
// hydist_gtsv_batched_noalloc: the Thomas solve of hydist_gtsv_batched with
// its forward-sweep scratch in a fixed device array of this library
// (HYDIST_GTSV_NOALLOC_MAX_ROWS rows of 8 bytes, reserved when the library's
// module is loaded on a device) instead of a cudaMalloc'd buffer, for callers
// that must not allocate device memory during a call. It allocates nothing:
// no cudaMalloc/cudaFree and no library that allocates. The first call on a
// device looks the array's address up (cudaGetSymbolAddress, once per device
// with that device current); that set-up call should come before any stream
// capture. Nothing in the scratch has to start at zero: every row a system
// reads is written by the same system's forward sweep first. The scratch is
// one per device, so two calls in flight on one device at the same time
// (different streams or host threads) race on it.
namespace hyd {

void set_last_error(const char* m);

__device__ __align__(256) double g_noalloc_w[HYDIST_GTSV_NOALLOC_MAX_ROWS];

// Thomas for systems that lie inside the packed rows [0, rows); a system
// outside them is left unsolved (offsets and lengths are device data, so
// this bound keeps every scratch access inside the fixed array).
template <class T>
__global__ void k_thomas_noalloc(const T* __restrict__ dl, const T* __restrict__ d,
                                 const T* __restrict__ du, const T* __restrict__ b, T* __restrict__ x,
                                 T* __restrict__ w, const int* __restrict__ off,
                                 const int* __restrict__ len, int nsys, int rows) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int o = off[s], n = len[s];
  if (n <= 0 || o < 0 || o > rows - n) return;
  const T* A = dl + o;
  const T* B = d + o;
  const T* C = du + o;
  const T* D = b + o;
  T* X = x + o;
  T* Wp = w + o;
  if (n == 1) {
    X[0] = D[0] / B[0];
    return;
  }
  T ap = -C[0] / B[0];
  T bp = D[0] / B[0];
  Wp[0] = ap;
  X[0] = bp;
  for (int i = 1; i < n - 1; ++i) {
    const T ep = A[i] * ap + B[i];
    ap = -C[i] / ep;
    bp = (D[i] - A[i] * bp) / ep;
    Wp[i] = ap;
    X[i] = bp;
  }
  T xr = (D[n - 1] - A[n - 1] * bp) / (B[n - 1] + A[n - 1] * ap);
  X[n - 1] = xr;
  for (int i = n - 2; i >= 0; --i) {
    xr = X[i] + Wp[i] * xr;
    X[i] = xr;
  }
}

}  // namespace hyd

namespace {
constexpr int kNoallocDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoallocDevices] = {};  // scratch address per device, set once
}  // namespace

extern "C" int hydist_gtsv_batched_noalloc(const void* dl, const void* d, const void* du,
                                           const void* b, void* x, const int32_t* offsets,
                                           const int32_t* lengths, int32_t nsys, int32_t rows,
                                           int32_t dtype, void* stream) {
  if (!dl || !d || !du || !b || !x || !offsets || !lengths || nsys < 0 || rows < 0) {
    hyd::set_last_error("hydist_gtsv_batched_noalloc: null pointer or negative size");
    return HYDIST_ERR_ARG;
  }
  if (dtype != 0 && dtype != 1) {
    hyd::set_last_error("hydist_gtsv_batched_noalloc: dtype must be 0 (FP64) or 1 (FP32)");
    return HYDIST_ERR_ARG;
  }
  if (rows > HYDIST_GTSV_NOALLOC_MAX_ROWS) {
    hyd::set_last_error(
        "hydist_gtsv_batched_noalloc: rows exceed the fixed scratch "
        "(HYDIST_GTSV_NOALLOC_MAX_ROWS); use hydist_gtsv_batched");
    return HYDIST_ERR_BUDGET;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    hyd::set_last_error("hydist_gtsv_batched_noalloc: cudaGetDevice failed");
    return HYDIST_ERR_CUDA;
  }
  if (dev < 0 || dev >= kNoallocDevices) {
    hyd::set_last_error("hydist_gtsv_batched_noalloc: device ordinal out of range");
    return HYDIST_ERR_ARG;
  }
  void* w = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, hyd::g_noalloc_w);
      if (e != cudaSuccess || !p) {
        hyd::set_last_error("hydist_gtsv_batched_noalloc: cudaGetSymbolAddress failed");
        return HYDIST_ERR_CUDA;
      }
      g_noalloc_ptr[dev] = p;
    }
    w = g_noalloc_ptr[dev];
  }
  if (nsys == 0 || rows == 0) return HYDIST_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int bs = 128, gs = (nsys + bs - 1) / bs;
  if (dtype == 0)
    hyd::k_thomas_noalloc<double><<<gs, bs, 0, st>>>(
        (const double*)dl, (const double*)d, (const double*)du, (const double*)b, (double*)x,
        (double*)w, offsets, lengths, nsys, rows);
  else
    hyd::k_thomas_noalloc<float><<<gs, bs, 0, st>>>(
        (const float*)dl, (const float*)d, (const float*)du, (const float*)b, (float*)x,
        (float*)w, offsets, lengths, nsys, rows);
  if (cudaGetLastError() != cudaSuccess) {
    hyd::set_last_error("hydist_gtsv_batched_noalloc: kernel launch failed");
    return HYDIST_ERR_CUDA;
  }
  return HYDIST_OK;
}
