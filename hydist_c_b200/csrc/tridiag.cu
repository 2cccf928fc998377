// tridiag.cu -- batched tridiagonal solver behind hydist_gtsv_batched.
//
// Replaces the reference's per-line solvers: tridiag()/tridiagSolver
// (UVZSolver_multithread.cpp:19-43, 78-109; serial Thomas, 32 redundant
// threads per line) and the SPIKE solver gtsv_spike_partial_diag_pivot_v1
// (gtsv.cpp:88-193, called per line with device-side allocation).
//
// Packed batch: system s occupies rows [off[s], off[s]+len[s]); dl of its
// first row and du of its last row are ignored.
//
// Three solvers, chosen per length band:
//   Thomas      one thread per system, in place in global memory (any length);
//   warp        one warp per system staged in shared memory, partition
//               method with a shuffle PCR of the 32 chunk separators
//               (systems up to GT_WARP_MAX rows);
//   CTA         one CTA of 256 or 512 threads per system, its rows staged
//               in shared memory by TMA bulk copies (the next system's while
//               one is solved, where two fit), partition method with a
//               shared-memory PCR (systems up to the shared memory of one
//               CTA, about 6000 FP64 / 12000 FP32 rows).
// A classification kernel files each system under its length band on the
// device; the bands' solvers then run over their lists. The autotuner times
// the feasible solvers per band on synthetic diagonally dominant batches and
// keeps the fastest (per device and dtype).
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "common.cuh"
#include "partsolve.cuh"

namespace hyd {

void set_last_error(const char* m);

constexpr int GT_NB = HYDIST_GTSV_BANDS;
constexpr int GT_WARPS = 4;      // warps per CTA of the warp solver
constexpr int GT_WARP_MAX = 512;  // longest system of the warp solver

// upper length bound of each band (the last is open)
__host__ __device__ inline int gt_band_hi(int b) {
  switch (b) {
    case 0: return 32;
    case 1: return 128;
    case 2: return 512;
    case 3: return 2048;
    case 4: return 4096;
    case 5: return 6144;
    default: return INT_MAX;
  }
}

// ---------------------------------------------------------------- Thomas
// The reference's algorithm (no pivoting): forward sweep with the modified
// super-diagonal in W and the modified right-hand side in X, then back
// substitution in X.
template <class T>
__device__ __forceinline__ void thomas_system(const T* A, const T* B, const T* C, const T* D, T* X,
                                              T* Wp, int n) {
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

// the systems of one band's list, one thread each
template <class T>
__global__ void k_thomas_list(const T* __restrict__ dl, const T* __restrict__ d,
                              const T* __restrict__ du, const T* __restrict__ b, T* __restrict__ x,
                              T* __restrict__ w, const int* __restrict__ off,
                              const int* __restrict__ len, const int* __restrict__ list,
                              const int* __restrict__ count) {
  const int cnt = *count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int s = list[i];
    const int o = off[s];
    thomas_system(dl + o, d + o, du + o, b + o, x + o, w + o, len[s]);
  }
}

// ---------------------------------------------------- diagonal pivoting
// Gaussian elimination with diagonal pivoting for systems that are not
// diagonally dominant: at each step the current diagonal (1x1 pivot) or the
// 2x2 block of the current and the next row is eliminated, by the
// Bunch-Kaufman criterion with kappa = (sqrt(5)-1)/2 (Bunch and Kaufman,
// Math. Comp. 31, 1977; the tridiagonal form of Erway and Marcia and of Chang
// et al., SC'12, which the reference's SPIKE tile solver,
// spike_kernel.hxx:119-376, also follows): the 1x1 pivot d' is taken when
// |d'| sigma >= kappa |c_k a_{k+1}|, sigma the largest magnitude of the
// entries coupling the next two rows. P holds the modified pivot of a row
// (for a 2x2 block: its first row's modified diagonal, its second row's
// determinant), F marks the second rows of 2x2 blocks, X the modified
// right-hand side and then the solution.
template <class T>
__device__ __forceinline__ void pivot_system(const T* A, const T* B, const T* C, const T* D, T* X,
                                             T* P, unsigned char* F, int n) {
  const T kappa = T(0.6180339887498949);
  T dk = B[0], rk = D[0];
  int k = 0;
  while (k < n) {
    F[k] = 0;
    if (k == n - 1) {
      P[k] = dk;
      X[k] = rk;
      break;
    }
    T sigma = fmax(fmax(fabs(C[k]), fabs(A[k + 1])), fabs(B[k + 1]));
    if (k + 2 < n) sigma = fmax(sigma, fmax(fabs(C[k + 1]), fabs(A[k + 2])));
    if (fabs(dk) * sigma >= kappa * fabs(C[k] * A[k + 1])) {
      P[k] = dk;
      X[k] = rk;
      const T l = A[k + 1] / dk;
      dk = B[k + 1] - l * C[k];
      rk = D[k + 1] - l * rk;
      k += 1;
    } else {
      const T det = dk * B[k + 1] - C[k] * A[k + 1];
      P[k] = dk;
      P[k + 1] = det;
      F[k + 1] = 1;
      X[k] = rk;
      X[k + 1] = D[k + 1];
      if (k + 2 < n) {
        // row k+2 minus A[k+2] times the block inverse's second row applied
        // to the block's right-hand sides ((B^-1)_22 = dk / det)
        const T l = A[k + 2] / det;
        rk = D[k + 2] - l * (dk * D[k + 1] - A[k + 1] * rk);
        dk = B[k + 2] - l * dk * C[k + 1];
      }
      k += 2;
    }
  }
  T xn = 0;  // x_{i+1}
  int i = n - 1;
  while (i >= 0) {
    if (F[i]) {
      // rows i-1, i: [[p, C[i-1]], [A[i], B[i]]] [x_{i-1}; x_i] = [r0; r1]
      const T p = P[i - 1], det = P[i];
      const T r0 = X[i - 1];
      const T r1 = X[i] - (i + 1 < n ? C[i] * xn : T(0));
      const T xi = (p * r1 - A[i] * r0) / det;
      const T xi1 = (B[i] * r0 - C[i - 1] * r1) / det;
      X[i] = xi;
      X[i - 1] = xi1;
      xn = xi1;
      i -= 2;
    } else {
      const T xi = (X[i] - (i + 1 < n ? C[i] * xn : T(0))) / P[i];
      X[i] = xi;
      xn = xi;
      i -= 1;
    }
  }
}

// the systems of one band's list, one thread each, with diagonal pivoting
// (P in the value scratch, F in the byte scratch, both at the system's rows)
template <class T>
__global__ void k_pivot_list(const T* __restrict__ dl, const T* __restrict__ d,
                             const T* __restrict__ du, const T* __restrict__ b, T* __restrict__ x,
                             T* __restrict__ w, unsigned char* __restrict__ flags,
                             const int* __restrict__ off, const int* __restrict__ len,
                             const int* __restrict__ list, const int* __restrict__ count) {
  const int cnt = *count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int s = list[i];
    const int o = off[s];
    pivot_system(dl + o, d + o, du + o, b + o, x + o, w + o, flags + o, len[s]);
  }
}

// ------------------------------------------------ refinement (FP64 systems)
// x32 -> x64 and the FP64 residual r = b - A x of the FP32 solution, rounded
// to FP32 as the right-hand side of the correction solve.
__global__ void k_gt_residual(const double* __restrict__ dl, const double* __restrict__ d,
                              const double* __restrict__ du, const double* __restrict__ b,
                              const float* __restrict__ x32, double* __restrict__ x,
                              float* __restrict__ r32, const int* __restrict__ off,
                              const int* __restrict__ len, int nsys) {
  const int s = blockIdx.x;
  if (s >= nsys) return;
  const int o = off[s], n = len[s];
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int g = o + q;
    const double xq = x32[g];
    double r = b[g] - d[g] * xq;
    if (q > 0) r -= dl[g] * (double)x32[g - 1];
    if (q + 1 < n) r -= du[g] * (double)x32[g + 1];
    x[g] = xq;
    r32[g] = (float)r;
  }
}

// x += the FP32 correction, in FP64
__global__ void k_gt_correct(double* __restrict__ x, const float* __restrict__ c32,
                             const int* __restrict__ off, const int* __restrict__ len, int nsys) {
  const int s = blockIdx.x;
  if (s >= nsys) return;
  const int o = off[s], n = len[s];
  for (int q = threadIdx.x; q < n; q += blockDim.x) x[o + q] += (double)c32[o + q];
}

// FP64 -> FP32 copies of a system's four arrays
// (array k at f + k * ld)
__global__ void k_gt_to_f32(const double* __restrict__ dl, const double* __restrict__ d,
                            const double* __restrict__ du, const double* __restrict__ b,
                            float* __restrict__ f, size_t rows, size_t ld) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < rows;
       r += (size_t)gridDim.x * blockDim.x) {
    f[r] = (float)dl[r];
    f[ld + r] = (float)d[r];
    f[2 * ld + r] = (float)du[r];
    f[3 * ld + r] = (float)b[r];
  }
}

// ------------------------------------------------- staged partition solvers
// Stages a system's rows into shared memory with asynchronous copies
// (cp.async): every thread's copies are in flight at once instead of one
// load latency per row. The caller synchronises the threads afterwards.
template <class T>
__device__ __forceinline__ void gt_load(const T* dl, const T* d, const T* du, const T* b, int o,
                                        int n, int S, T* rA, T* rB, T* rC, T* rD, int t0, int dt) {
  for (PartStrideIdx it(t0, dt, S); it.q < n; it.next(dt)) {
    const int i = it.q, q = it.idx();
    if (i > 0) __pipeline_memcpy_async(&rA[q], &dl[o + i], sizeof(T));
    else rA[q] = T(0);
    __pipeline_memcpy_async(&rB[q], &d[o + i], sizeof(T));
    if (i < n - 1) __pipeline_memcpy_async(&rC[q], &du[o + i], sizeof(T));
    else rC[q] = T(0);
    __pipeline_memcpy_async(&rD[q], &b[o + i], sizeof(T));
  }
  __pipeline_commit();
  __pipeline_wait_prior(0);
}

// ------------------------------------------ bulk-staged partition solver
// One system per CTA of NT threads. Thread 0 stages the system's rows with
// TMA bulk copies (cp.async.bulk, completion counted on an mbarrier) into an
// unpadded layout; the few rows at either end that are not 16-byte aligned
// in global memory are read with plain loads. With NBUF = 2 the next
// system's rows are fetched while the current one is solved. The chunk
// length S is odd, so the threads' walks over their chunks (a stride of S
// rows between threads) fall on distinct shared-memory banks.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// the index of row 0 of a system at offset o within an array's region: the
// region starts 16-byte aligned and the rows from a0 (o rounded up to 16
// bytes) on land 16-byte aligned
template <class T>
__device__ __forceinline__ int bulk_pad(int o) {
  constexpr int E = 16 / sizeof(T);
  const int d = (E - o % E) % E;  // a0 - o
  return (E - d) % E;
}

// elements of one array's region for systems of up to nmax rows
template <class T>
__host__ __device__ inline int bulk_region(int nmax) {
  constexpr int E = 16 / sizeof(T);
  return (nmax + 2 * E + E - 1) / E * E;
}

// the odd chunk length of a system of n rows on NT threads (at least 3)
__device__ __forceinline__ int bulk_chunk(int n, int NT) {
  int S = (n + NT - 1) / NT;
  if (S < 3) S = 3;
  return S | 1;
}

// waits of the staging barrier before a CTA gives a system up (each try
// suspends the thread for a while; a stalled copy is reported, not waited
// for without end)
constexpr long GT_WAIT_TRIES = 1L << 22;

template <class T, int NT, int NBUF>
__global__ void __launch_bounds__(NT) k_gtsv_bulk(const T* __restrict__ dl, const T* __restrict__ d,
                                                  const T* __restrict__ du, const T* __restrict__ b,
                                                  T* __restrict__ x, const int* __restrict__ off,
                                                  const int* __restrict__ len,
                                                  const int* __restrict__ list,
                                                  const int* __restrict__ count, int region,
                                                  int* __restrict__ stalled) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // NBUF barriers
  auto& sh = *reinterpret_cast<PartCtaShared<T, NT>*>(smem_raw + 128);
  T* bufs = reinterpret_cast<T*>(smem_raw + 128 + (sizeof(PartCtaShared<T, NT>) + 127) / 128 * 128);
  constexpr int E = 16 / sizeof(T);
  const int tid = threadIdx.x;
  const int cnt = *count;
  const T* src[4] = {dl, d, du, b};
  // thread 0: the bulk copies of system list[i] into buffer k
  auto issue = [&](int i, int k) {
    const int sys = list[i];
    const int o = off[sys], n = len[sys];
    const int a0 = (o + E - 1) / E * E, a1 = (o + n) / E * E;
    T* base = bufs + (size_t)k * 4 * region + bulk_pad<T>(o);
    if (a1 > a0) {
      const unsigned bytes = (unsigned)((a1 - a0) * sizeof(T));
      mbar_arrive_expect(&bar[k], 4 * bytes);
      for (int a = 0; a < 4; ++a) bulk_g2s(base + (size_t)a * region + (a0 - o), src[a] + a0, bytes, &bar[k]);
    } else {
      mbar_arrive_expect(&bar[k], 0);
    }
  };
  if (tid == 0) {
    for (int k = 0; k < NBUF; ++k) mbar_init(&bar[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < cnt) issue(blockIdx.x, 0);
  unsigned phase = 0;  // bit k: the parity of buffer k's next completion
  int it = 0;
  for (int i = blockIdx.x; i < cnt; i += gridDim.x, ++it) {
    const int k = NBUF == 2 ? (it & 1) : 0;
    const int sys = list[i];
    const int o = off[sys], n = len[sys];
    // wait for the rows (bounded)
    bool ok = false;
    for (long t = 0; t < GT_WAIT_TRIES && !ok; ++t) ok = mbar_try_wait(&bar[k], (phase >> k) & 1u);
    if (!__syncthreads_and(ok)) {
      // a copy that never completed: record it, give the copy in flight
      // (the only one: the next system's is issued after this test) one
      // more bounded wait, and leave the CTA's remaining systems unsolved;
      // the call reports HYDIST_ERR_TIMEOUT for this batch
      if (tid == 0) {
        atomicExch(stalled, 1);
        bool done = false;
        for (long t = 0; t < GT_WAIT_TRIES && !done; ++t) done = mbar_try_wait(&bar[k], (phase >> k) & 1u);
      }
      __syncthreads();
      return;
    }
    phase ^= 1u << k;
    const int inext = i + gridDim.x;
    if (NBUF == 2 && tid == 0 && inext < cnt) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(inext, k ^ 1);
    }
    T* rA = bufs + (size_t)k * 4 * region + bulk_pad<T>(o);
    T* rB = rA + region;
    T* rC = rB + region;
    T* rD = rC + region;
    // the rows outside the aligned bulk part
    const int a0 = (o + E - 1) / E * E, a1 = (o + n) / E * E;
    const int head = min(a0 - o, n), tail0 = max(a1 - o, head);
    for (int q = tid; q < head + (n - tail0); q += NT) {
      const int r = q < head ? q : tail0 + (q - head);
      rA[r] = dl[o + r];
      rB[r] = d[o + r];
      rC[r] = du[o + r];
      rD[r] = b[o + r];
    }
    __syncthreads();
    // ---- partition solve in place: forward per chunk, separators by PCR
    const int S = bulk_chunk(n, NT), P = max(1, n / S);
    const int q0 = tid * S;
    const int nu = tid < P ? (tid == P - 1 ? n - q0 : S) : 0;
    T sep[4] = {0, 1, 0, 0};
    T cp = 0, yp = 0, vp = 0, Pk = 1, fy = 0, fv = 0;
    for (int s = 0; s < nu; ++s) {
      const int q = q0 + s;
      const T A = q > 0 ? rA[q] : T(0), B = rB[q], C = q + 1 < n ? rC[q] : T(0), Dv = rD[q];
      if (s == nu - 1) {
        sep[0] = A;
        sep[1] = B;
        sep[2] = C;
        sep[3] = Dv;
      } else {
        if (s == 0) {
          const T m = T(1) / B;
          cp = C * m;
          yp = Dv * m;
          vp = -A * m;
        } else {
          const T m = T(1) / (B - A * cp);
          yp = (Dv - A * yp) * m;
          vp = -A * vp * m;
          cp = C * m;
        }
        rC[q] = cp;
        rD[q] = yp;
        rA[q] = vp;
        fy += Pk * yp;
        fv += Pk * vp;
        Pk *= -cp;
      }
    }
    sh.tri[0][tid] = fy;
    sh.tri[1][tid] = fv;
    sh.tri[2][tid] = Pk;
    __syncthreads();
    T ra = 0, rb = 1, rc = 0, rd = 0;
    if (tid < P) {
      T yF = 0, vF = 0, wF = 0;
      if (tid + 1 < P) {
        yF = sh.tri[0][tid + 1];
        vF = sh.tri[1][tid + 1];
        wF = sh.tri[2][tid + 1];
      }
      ra = sep[0] * vp;
      rb = sep[1] - sep[0] * cp + sep[2] * vF;
      rc = sep[2] * wF;
      rd = sep[3] - sep[0] * yp - sep[2] * yF;
    }
    for (int st = 1; st < P; st <<= 1) {
      sh.red[0][tid] = ra;
      sh.red[1][tid] = rb;
      sh.red[2][tid] = rc;
      sh.red[3][tid] = rd;
      __syncthreads();
      T am = 0, bm = 1, cm = 0, dm = 0, an = 0, bn = 1, cn = 0, dn = 0;
      if (tid < P && tid - st >= 0) {
        am = sh.red[0][tid - st];
        bm = sh.red[1][tid - st];
        cm = sh.red[2][tid - st];
        dm = sh.red[3][tid - st];
      }
      if (tid + st < P) {
        an = sh.red[0][tid + st];
        bn = sh.red[1][tid + st];
        cn = sh.red[2][tid + st];
        dn = sh.red[3][tid + st];
      }
      __syncthreads();
      const T k1 = ra / bm, k2 = rc / bn;
      const T na = -am * k1, nc = -cn * k2;
      const T nb = rb - cm * k1 - an * k2;
      const T nd = rd - dm * k1 - dn * k2;
      ra = na;
      rb = nb;
      rc = nc;
      rd = nd;
    }
    sh.xsep[tid] = rd / rb;
    __syncthreads();
    if (tid < P) {
      const T xl = tid > 0 ? sh.xsep[tid - 1] : T(0), xr = sh.xsep[tid];
      rD[q0 + nu - 1] = xr;
      T xn = xr;
      for (int t = nu - 2; t >= 0; --t) {
        const int q = q0 + t;
        const T xq = rD[q] + rA[q] * xl - rC[q] * xn;
        rD[q] = xq;
        xn = xq;
      }
    }
    __syncthreads();
    for (int q = tid; q < n; q += NT) x[o + q] = rD[q];
    __syncthreads();  // the buffer is free
    if (NBUF == 1 && tid == 0 && inext < cnt) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(inext, 0);
    }
  }
}

template <class T>
__global__ void __launch_bounds__(GT_WARPS * 32) k_gtsv_warp(
    const T* __restrict__ dl, const T* __restrict__ d, const T* __restrict__ du,
    const T* __restrict__ b, T* __restrict__ x, const int* __restrict__ off,
    const int* __restrict__ len, const int* __restrict__ list, const int* __restrict__ count,
    int slice) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T* base = reinterpret_cast<T*>(smem_raw) + (size_t)warp * 4 * slice;
  const int cnt = *count;
  for (int i = blockIdx.x * GT_WARPS + warp; i < cnt; i += gridDim.x * GT_WARPS) {
    const int s = list[i];
    const int o = off[s], n = len[s];
    const PartGeom g = part_geom(n, 32);
    T* rA = base;
    T* rB = rA + g.stride;
    T* rC = rB + g.stride;
    T* rD = rC + g.stride;
    gt_load(dl, d, du, b, o, n, g.S, rA, rB, rC, rD, lane, 32);
    __syncwarp();
    part_solve_warp<T>(rA, rB, rC, rD, g, n, lane);
    for (PartStrideIdx it(lane, 32, g.S); it.q < n; it.next(32)) x[o + it.q] = rD[it.idx()];
    __syncwarp();
  }
}

// Files system s under its length band (empty systems under none). Also
// counts[GT_NB] = the packed extent max(off + len), counts[GT_NB + 1] = 1 if
// a system has a negative offset (the batch is then refused).
__global__ void k_gt_classify(const int* __restrict__ off, const int* __restrict__ len, int nsys,
                              int* __restrict__ lists, int* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const int n = len[s];
  if (n <= 0) return;
  const int o = off[s];
  if (o < 0 || o > INT_MAX - n) {
    counts[GT_NB + 1] = 1;
    return;
  }
  atomicMax(&counts[GT_NB], o + n);
  int b = 0;
  while (b < GT_NB - 1 && n > gt_band_hi(b)) ++b;
  const int idx = atomicAdd(&counts[b], 1);
  lists[(size_t)b * nsys + idx] = s;
}

// diagonally dominant synthetic systems for the autotuner (a counter hash)
__device__ __forceinline__ double gt_unit(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return (double)(k >> 11) * (1.0 / 9007199254740992.0);
}

template <class T>
__global__ void k_gt_synth(T* dl, T* d, T* du, T* b, size_t rows, unsigned seed) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < rows;
       r += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long k = ((unsigned long long)seed << 40) ^ (r * 4);
    const double a = 2 * gt_unit(k) - 1, c = 2 * gt_unit(k + 1) - 1;
    dl[r] = (T)a;
    du[r] = (T)c;
    d[r] = (T)(fabs(a) + fabs(c) + 0.1 + 0.9 * gt_unit(k + 2));
    b[r] = (T)(2 * gt_unit(k + 3) - 1);
  }
}

}  // namespace hyd

// ====================================================================== host
namespace {

using hyd::GT_NB;

struct DevScratch {
  void* w = nullptr;  // Thomas forward-sweep / pivoting scratch (rows x 8 B)
  size_t w_bytes = 0;
  unsigned char* flags = nullptr;  // pivoting: 2x2 block marks (rows x 1 B)
  size_t flags_bytes = 0;
  float* f32 = nullptr;  // refinement: FP32 copies of the systems and x (rows x 5 x 4 B)
  size_t f32_bytes = 0;
  int* lists = nullptr;  // GT_NB x nsys
  size_t lists_cap = 0;  // systems
  int* counts = nullptr;  // GT_NB
};

struct DevInfo {
  int nsm = 0, optin = 0;
  bool init = false;
  int table[2][GT_NB] = {};  // autotuned solver per dtype and band (0: not tuned)
  DevScratch scr;
  // the bands of a batch run side by side: one stream per band, forked from
  // the caller's stream and joined back (created on first use, kept)
  cudaStream_t band_st[GT_NB] = {};
  cudaEvent_t fork = nullptr, join[GT_NB] = {};
  bool streams = false;
};

std::mutex g_mu;
DevInfo g_dev[64];

DevInfo* dev_info(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  DevInfo& D = g_dev[dev];
  if (!D.init) {
    cudaDeviceGetAttribute(&D.nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&D.optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    D.init = true;
  }
  return &D;
}

// shared memory of the bulk-staged CTA solver for systems of up to nmax
// rows with nbuf row buffers (monotonic in nmax)
template <class T, int NT>
size_t cta_smem(int nmax, int nbuf = 1) {
  return 128 + (sizeof(hyd::PartCtaShared<T, NT>) + 127) / 128 * 128 +
         (size_t)nbuf * 4 * hyd::bulk_region<T>(nmax) * sizeof(T);
}

template <class T>
size_t warp_smem(int nmax) {
  return (size_t)hyd::GT_WARPS * 4 * sizeof(T) * (size_t)hyd::part_stride_bound(nmax, 32);
}

// longest system the CTA solver with NT threads takes on this device
template <class T, int NT>
int cta_max_rows(const DevInfo& D) {
  int lo = 2, hi = 1 << 16;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (cta_smem<T, NT>(mid) <= (size_t)D.optin) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct Caps {
  int cta128, cta256, cta512;  // longest systems of the three CTA tiles
};

template <class T>
Caps caps_of(const DevInfo& D) {
  return Caps{cta_max_rows<T, 128>(D), cta_max_rows<T, 256>(D), cta_max_rows<T, 512>(D)};
}

bool feasible(int algo, int band, const Caps& c) {
  const int hi = hyd::gt_band_hi(band);
  if (algo == HYDIST_GTSV_THOMAS || algo == HYDIST_GTSV_PIVOT) return true;
  if (algo == HYDIST_GTSV_WARP) return hi <= hyd::GT_WARP_MAX;
  if (algo == HYDIST_GTSV_PARTITION) return hi <= c.cta256;
  if (algo == HYDIST_GTSV_PARTITION_512) return hi <= c.cta512;
  if (algo == HYDIST_GTSV_PARTITION_128) return hi <= c.cta128;
  return false;
}

// solver of a band when nothing was tuned: warp for short systems, the
// 512-thread tile for long ones that fit, the 256-thread tile beyond,
// Thomas for what fits no shared memory
int default_algo(int band, const Caps& c) {
  if (feasible(HYDIST_GTSV_WARP, band, c)) return HYDIST_GTSV_WARP;
  if (feasible(HYDIST_GTSV_PARTITION_512, band, c)) return HYDIST_GTSV_PARTITION_512;
  if (feasible(HYDIST_GTSV_PARTITION, band, c)) return HYDIST_GTSV_PARTITION;
  return HYDIST_GTSV_THOMAS;
}

// Resident CTAs per SM of `kernel` with NT threads and `smem` bytes of
// dynamic shared memory on the current device, its shared-memory limit
// raised to the opt-in maximum; queried once per (device, kernel, smem),
// since a batched solve launches the same few configurations every call.
template <class K>
int resident_ctas(K kernel, int nt, size_t smem, int optin) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, size_t>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(dev, (const void*)kernel, smem);
  std::lock_guard<std::mutex> lk(mu);
  const auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, smem) != cudaSuccess)
    return 0;
  cache[key] = per_sm;
  return per_sm;
}

template <class T, int NT, int NBUF>
int launch_bulk(int nmax, const T* dl, const T* d, const T* du, const T* b, T* x, const int* off,
                const int* len, const int* list, const int* count, int* stalled, int nsys_band,
                const DevInfo& D, cudaStream_t st) {
  const size_t smem = cta_smem<T, NT>(nmax, NBUF);
  const int per_sm = resident_ctas(hyd::k_gtsv_bulk<T, NT, NBUF>, NT, smem, D.optin);
  if (per_sm < 1) return HYDIST_ERR_CUDA;
  const int grid = std::min(nsys_band, per_sm * D.nsm);
  hyd::k_gtsv_bulk<T, NT, NBUF><<<grid, NT, smem, st>>>(dl, d, du, b, x, off, len, list, count,
                                                         hyd::bulk_region<T>(nmax), stalled);
  return HYDIST_OK;
}

// CTAs of the bulk-staged solver resident per SM with nbuf row buffers
template <class T, int NT>
int bulk_per_sm(int nmax, int nbuf, const DevInfo& D) {
  const size_t smem = cta_smem<T, NT>(nmax, nbuf);
  if (smem > (size_t)D.optin) return 0;
  return nbuf == 2 ? resident_ctas(hyd::k_gtsv_bulk<T, NT, 2>, NT, smem, D.optin)
                   : resident_ctas(hyd::k_gtsv_bulk<T, NT, 1>, NT, smem, D.optin);
}

// the CTA solver: the next system's rows are staged while one is solved
// where the second buffer costs no resident CTA
template <class T, int NT>
int launch_cta(int nmax, const T* dl, const T* d, const T* du, const T* b, T* x, const int* off,
               const int* len, const int* list, const int* count, int* stalled, int nsys_band,
               const DevInfo& D, cudaStream_t st) {
  if (bulk_per_sm<T, NT>(nmax, 2, D) >= std::max(1, bulk_per_sm<T, NT>(nmax, 1, D)))
    return launch_bulk<T, NT, 2>(nmax, dl, d, du, b, x, off, len, list, count, stalled, nsys_band, D, st);
  return launch_bulk<T, NT, 1>(nmax, dl, d, du, b, x, off, len, list, count, stalled, nsys_band, D, st);
}

template <class T>
int launch_band(int algo, int band, const T* dl, const T* d, const T* du, const T* b, T* x, T* w,
                unsigned char* flags, const int* off, const int* len, const int* list,
                const int* count, int* stalled, int nsys_band, const DevInfo& D, cudaStream_t st) {
  if (nsys_band <= 0) return HYDIST_OK;
  const int hi = hyd::gt_band_hi(band);
  int rc = HYDIST_OK;
  if (algo == HYDIST_GTSV_PIVOT) {
    const int bs = 128;
    const int grid = std::min((nsys_band + bs - 1) / bs, 8 * D.nsm);
    hyd::k_pivot_list<T><<<grid, bs, 0, st>>>(dl, d, du, b, x, w, flags, off, len, list, count);
  } else if (algo == HYDIST_GTSV_PARTITION_128) {
    rc = launch_cta<T, 128>(hi, dl, d, du, b, x, off, len, list, count, stalled, nsys_band, D, st);
  } else if (algo == HYDIST_GTSV_PARTITION) {
    rc = launch_cta<T, 256>(hi, dl, d, du, b, x, off, len, list, count, stalled, nsys_band, D, st);
  } else if (algo == HYDIST_GTSV_PARTITION_512) {
    rc = launch_cta<T, 512>(hi, dl, d, du, b, x, off, len, list, count, stalled, nsys_band, D, st);
  } else if (algo == HYDIST_GTSV_WARP) {
    const int nmax = std::min(hi, hyd::GT_WARP_MAX);
    const int slice = hyd::part_stride_bound(nmax, 32);
    const size_t smem = warp_smem<T>(nmax);
    const int per_sm = resident_ctas(hyd::k_gtsv_warp<T>, hyd::GT_WARPS * 32, smem, D.optin);
    if (per_sm < 1) return HYDIST_ERR_CUDA;
    const int grid = std::min((nsys_band + hyd::GT_WARPS - 1) / hyd::GT_WARPS, per_sm * D.nsm);
    hyd::k_gtsv_warp<T><<<grid, hyd::GT_WARPS * 32, smem, st>>>(dl, d, du, b, x, off, len, list,
                                                                  count, slice);
  } else {
    const int bs = 128;
    const int grid = std::min((nsys_band + bs - 1) / bs, 8 * D.nsm);
    hyd::k_thomas_list<T><<<grid, bs, 0, st>>>(dl, d, du, b, x, w, off, len, list, count);
  }
  if (rc != HYDIST_OK) return rc;
  return cudaGetLastError() == cudaSuccess ? HYDIST_OK : HYDIST_ERR_CUDA;
}

int ensure_scratch(DevScratch& s, size_t w_bytes, size_t nsys, size_t flag_bytes = 0) {
  if (w_bytes > 0 && s.w_bytes < w_bytes) {
    if (s.w) cudaFree(s.w);
    s.w = nullptr;
    s.w_bytes = 0;
    if (cudaMalloc(&s.w, w_bytes + 256) != cudaSuccess) return HYDIST_ERR_OOM;
    s.w_bytes = w_bytes;
  }
  if (flag_bytes > 0 && s.flags_bytes < flag_bytes) {
    if (s.flags) cudaFree(s.flags);
    s.flags = nullptr;
    s.flags_bytes = 0;
    if (cudaMalloc(&s.flags, flag_bytes + 256) != cudaSuccess) return HYDIST_ERR_OOM;
    s.flags_bytes = flag_bytes;
  }
  if (s.lists_cap < nsys) {
    if (s.lists) cudaFree(s.lists);
    s.lists = nullptr;
    s.lists_cap = 0;
    if (cudaMalloc(&s.lists, (size_t)GT_NB * nsys * sizeof(int)) != cudaSuccess) return HYDIST_ERR_OOM;
    s.lists_cap = nsys;
  }
  // band sizes, packed extent, offset check, and a flag that stays set
  // until read: a CTA solver gave a system up (its staging never completed)
  if (!s.counts) {
    if (cudaMalloc(&s.counts, (GT_NB + 3) * sizeof(int)) != cudaSuccess) return HYDIST_ERR_OOM;
    if (cudaMemset(s.counts, 0, (GT_NB + 3) * sizeof(int)) != cudaSuccess) return HYDIST_ERR_CUDA;
  }
  return HYDIST_OK;
}

// the per-band streams and events of a device (false if they cannot be made:
// the bands then run one after another on the caller's stream)
bool band_streams(DevInfo& D) {
  if (D.streams) return true;
  for (int k = 0; k < GT_NB; ++k) {
    if (!D.band_st[k] && cudaStreamCreateWithFlags(&D.band_st[k], cudaStreamNonBlocking) != cudaSuccess)
      return false;
    if (!D.join[k] && cudaEventCreateWithFlags(&D.join[k], cudaEventDisableTiming) != cudaSuccess)
      return false;
  }
  if (!D.fork && cudaEventCreateWithFlags(&D.fork, cudaEventDisableTiming) != cudaSuccess) return false;
  D.streams = true;
  return true;
}

// one batched solve with a given solver per band (table[b])
template <class T>
int solve_batch(const T* dl, const T* d, const T* du, const T* b, T* x, const int* off,
                const int* len, int nsys, const int table[GT_NB], DevInfo& D, cudaStream_t st) {
  int rc = ensure_scratch(D.scr, 0, (size_t)nsys);
  if (rc != HYDIST_OK) return rc;
  if (cudaMemsetAsync(D.scr.counts, 0, (GT_NB + 2) * sizeof(int), st) != cudaSuccess)
    return HYDIST_ERR_CUDA;
  hyd::k_gt_classify<<<(nsys + 255) / 256, 256, 0, st>>>(off, len, nsys, D.scr.lists, D.scr.counts);
  // band sizes, packed extent and the offset check in one synchronisation
  int counts[GT_NB + 3];
  if (cudaMemcpyAsync(counts, D.scr.counts, sizeof(counts), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return HYDIST_ERR_CUDA;
  if (counts[GT_NB + 1]) return HYDIST_ERR_ARG;
  // the CTA solvers stage rows with bulk copies, which need 16-byte aligned
  // arrays; misaligned ones go to Thomas
  int tab[GT_NB];
  const bool aligned =
      (((uintptr_t)dl | (uintptr_t)d | (uintptr_t)du | (uintptr_t)b) & 15) == 0;
  for (int bnd = 0; bnd < GT_NB; ++bnd)
    tab[bnd] = (!aligned && (table[bnd] == HYDIST_GTSV_PARTITION ||
                             table[bnd] == HYDIST_GTSV_PARTITION_512 ||
                             table[bnd] == HYDIST_GTSV_PARTITION_128))
                   ? HYDIST_GTSV_THOMAS
                   : table[bnd];
  table = tab;
  bool thomas = false, pivot = false;
  for (int bnd = 0; bnd < GT_NB; ++bnd) {
    thomas |= counts[bnd] > 0 && table[bnd] == HYDIST_GTSV_THOMAS;
    pivot |= counts[bnd] > 0 && table[bnd] == HYDIST_GTSV_PIVOT;
  }
  if (thomas || pivot) {
    rc = ensure_scratch(D.scr, (size_t)counts[GT_NB] * sizeof(T), (size_t)nsys,
                        pivot ? (size_t)counts[GT_NB] : 0);
    if (rc != HYDIST_OK) return rc;
  }
  bool staged = false;  // a bulk-staged CTA solver ran
  // the bands' solves are independent (disjoint systems, per-band lists,
  // per-system scratch): each non-empty band on its own stream, so that the
  // short bands' launches and the long bands' tails overlap
  int nonempty = 0;
  for (int bnd = 0; bnd < GT_NB; ++bnd) nonempty += counts[bnd] > 0;
  const bool side = nonempty > 1 && band_streams(D);
  if (side && cudaEventRecord(D.fork, st) != cudaSuccess) return HYDIST_ERR_CUDA;
  for (int bnd = 0; bnd < GT_NB; ++bnd) {
    if (counts[bnd] == 0) continue;
    cudaStream_t bs = st;
    if (side) {
      bs = D.band_st[bnd];
      if (cudaStreamWaitEvent(bs, D.fork, 0) != cudaSuccess) return HYDIST_ERR_CUDA;
    }
    rc = launch_band<T>(table[bnd], bnd, dl, d, du, b, x, (T*)D.scr.w, D.scr.flags, off, len,
                        D.scr.lists + (size_t)bnd * nsys, D.scr.counts + bnd,
                        D.scr.counts + GT_NB + 2, counts[bnd], D, bs);
    if (side && (cudaEventRecord(D.join[bnd], bs) != cudaSuccess ||
                 cudaStreamWaitEvent(st, D.join[bnd], 0) != cudaSuccess))
      return HYDIST_ERR_CUDA;
    if (rc != HYDIST_OK) return rc;
    staged |= table[bnd] == HYDIST_GTSV_PARTITION || table[bnd] == HYDIST_GTSV_PARTITION_512 ||
              table[bnd] == HYDIST_GTSV_PARTITION_128;
  }
  if (staged) {
    // a CTA whose staging copy never completed left systems unsolved: read
    // its flag now, so that this batch, not a later one, reports it
    int flag = 0;
    if (cudaMemcpyAsync(&flag, D.scr.counts + GT_NB + 2, sizeof(int), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return HYDIST_ERR_CUDA;
    if (flag) {
      cudaMemsetAsync(D.scr.counts + GT_NB + 2, 0, sizeof(int), st);
      return HYDIST_ERR_TIMEOUT;
    }
  }
  return HYDIST_OK;
}

template <class T>
int autotune(DevInfo& D, int dtype, cudaStream_t st) {
  const Caps caps = caps_of<T>(D);
  for (int bnd = 0; bnd < GT_NB; ++bnd) {
    int cands[5], nc = 0;
    for (int a : {HYDIST_GTSV_THOMAS, HYDIST_GTSV_PARTITION, HYDIST_GTSV_PARTITION_512,
                  HYDIST_GTSV_WARP, HYDIST_GTSV_PARTITION_128})
      if (feasible(a, bnd, caps)) cands[nc++] = a;
    if (nc == 1) {
      D.table[dtype][bnd] = cands[0];
      continue;
    }
    // synthetic batch: lengths log-uniform within the band, about 4M rows
    const int lo = bnd == 0 ? 1 : hyd::gt_band_hi(bnd - 1) + 1;
    const int hi = std::min(hyd::gt_band_hi(bnd), 1 << 16);
    std::vector<int> off, len;
    size_t rows = 0;
    unsigned long long r = 0x9e3779b97f4a7c15ULL * (bnd + 1);
    while (rows < (4u << 20) && (int)len.size() < 16384) {
      r = r * 6364136223846793005ULL + 1442695040888963407ULL;
      const double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
      const int n = std::max(lo, std::min(hi, (int)std::exp(std::log((double)lo) +
                                                            u * (std::log((double)hi) - std::log((double)lo)))));
      off.push_back((int)rows);
      len.push_back(n);
      rows += n;
    }
    const int ns = (int)len.size();
    T *dl = nullptr, *dd = nullptr, *du = nullptr, *bb = nullptr, *xx = nullptr;
    int *doff = nullptr, *dlen = nullptr;
    bool ok = cudaMalloc(&dl, rows * sizeof(T)) == cudaSuccess &&
              cudaMalloc(&dd, rows * sizeof(T)) == cudaSuccess &&
              cudaMalloc(&du, rows * sizeof(T)) == cudaSuccess &&
              cudaMalloc(&bb, rows * sizeof(T)) == cudaSuccess &&
              cudaMalloc(&xx, rows * sizeof(T)) == cudaSuccess &&
              cudaMalloc(&doff, ns * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&dlen, ns * sizeof(int)) == cudaSuccess;
    int rc = ok ? HYDIST_OK : HYDIST_ERR_OOM;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ok) {
      cudaMemcpyAsync(doff, off.data(), ns * sizeof(int), cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(dlen, len.data(), ns * sizeof(int), cudaMemcpyHostToDevice, st);
      hyd::k_gt_synth<T><<<4 * D.nsm, 256, 0, st>>>(dl, dd, du, bb, rows, 77u + bnd);
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      float best = 1e30f;
      int best_a = cands[0];
      for (int c = 0; c < nc && rc == HYDIST_OK; ++c) {
        int table[GT_NB];
        for (int k = 0; k < GT_NB; ++k) table[k] = cands[c];
        float tmin = 1e30f;
        for (int rep = 0; rep < 4 && rc == HYDIST_OK; ++rep) {
          cudaEventRecord(e0, st);
          rc = solve_batch<T>(dl, dd, du, bb, xx, doff, dlen, ns, table, D, st);
          cudaEventRecord(e1, st);
          cudaEventSynchronize(e1);
          float ms = 0;
          cudaEventElapsedTime(&ms, e0, e1);
          if (rep > 0) tmin = std::min(tmin, ms);  // the first run warms up
        }
        if (tmin < best) {
          best = tmin;
          best_a = cands[c];
        }
      }
      D.table[dtype][bnd] = best_a;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    for (void* p : {(void*)dl, (void*)dd, (void*)du, (void*)bb, (void*)xx, (void*)doff, (void*)dlen})
      if (p) cudaFree(p);
    if (rc != HYDIST_OK) return rc;
  }
  return cudaGetLastError() == cudaSuccess ? HYDIST_OK : HYDIST_ERR_CUDA;
}

}  // namespace

extern "C" int hydist_gtsv_autotune(int32_t dtype, void* stream, int32_t* algo_per_band) {
  if (dtype != 0 && dtype != 1) {
    hyd::set_last_error("hydist_gtsv_autotune: dtype must be 0 (FP64) or 1 (FP32)");
    return HYDIST_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return HYDIST_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DevInfo* D = dev_info(dev);
  if (!D) return HYDIST_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = dtype == 0 ? autotune<double>(*D, 0, st) : autotune<float>(*D, 1, st);
  if (rc != HYDIST_OK) {
    hyd::set_last_error("hydist_gtsv_autotune: a CUDA call failed");
    return rc;
  }
  if (algo_per_band)
    for (int b = 0; b < GT_NB; ++b) algo_per_band[b] = D->table[dtype][b];
  return HYDIST_OK;
}

extern "C" int hydist_gtsv_band_bounds(int32_t* hi) {
  if (!hi) return HYDIST_ERR_ARG;
  for (int b = 0; b < GT_NB; ++b) hi[b] = hyd::gt_band_hi(b);
  return HYDIST_OK;
}

extern "C" int hydist_gtsv_batched(const void* dl, const void* d, const void* du, const void* b,
                                   void* x, const int32_t* offsets, const int32_t* lengths,
                                   int32_t nsys, int32_t dtype, int32_t algo, void* stream) {
  if (!dl || !d || !du || !b || !x || !offsets || !lengths || nsys < 0) {
    hyd::set_last_error("hydist_gtsv_batched: null pointer or negative count");
    return HYDIST_ERR_ARG;
  }
  if (dtype != 0 && dtype != 1) {
    hyd::set_last_error("hydist_gtsv_batched: dtype must be 0 (FP64) or 1 (FP32)");
    return HYDIST_ERR_ARG;
  }
  if (algo < HYDIST_GTSV_AUTO || algo > HYDIST_GTSV_PIVOT) {
    hyd::set_last_error("hydist_gtsv_batched: unknown algo");
    return HYDIST_ERR_ARG;
  }
  if (nsys == 0) return HYDIST_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return HYDIST_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  DevInfo* D = dev_info(dev);
  if (!D) return HYDIST_ERR_ARG;
  const Caps caps = dtype == 0 ? caps_of<double>(*D) : caps_of<float>(*D);
  int table[GT_NB];
  for (int bnd = 0; bnd < GT_NB; ++bnd) {
    int a = algo;
    if (a == HYDIST_GTSV_AUTO) a = D->table[dtype][bnd] ? D->table[dtype][bnd] : default_algo(bnd, caps);
    // a solver that cannot take the band's lengths hands it to the next
    // more general one: warp -> 512-thread tile -> 256-thread tile -> Thomas
    if (a == HYDIST_GTSV_PARTITION_128 && !feasible(a, bnd, caps)) a = HYDIST_GTSV_PARTITION;
    if (a == HYDIST_GTSV_WARP && !feasible(a, bnd, caps)) a = HYDIST_GTSV_PARTITION_512;
    if (a == HYDIST_GTSV_PARTITION_512 && !feasible(a, bnd, caps)) a = HYDIST_GTSV_PARTITION;
    if (a == HYDIST_GTSV_PARTITION && !feasible(a, bnd, caps)) a = HYDIST_GTSV_THOMAS;
    table[bnd] = a;
  }
  int rc;
  if (dtype == 0) {
    rc = solve_batch<double>((const double*)dl, (const double*)d, (const double*)du,
                             (const double*)b, (double*)x, offsets, lengths, nsys, table, *D, st);
  } else {
    rc = solve_batch<float>((const float*)dl, (const float*)d, (const float*)du, (const float*)b,
                            (float*)x, offsets, lengths, nsys, table, *D, st);
  }
  if (rc == HYDIST_ERR_ARG) hyd::set_last_error("hydist_gtsv_batched: a system has a negative offset");
  else if (rc == HYDIST_ERR_TIMEOUT)
    hyd::set_last_error("hydist_gtsv_batched: a CTA solver gave up waiting for a system's rows "
                        "in shared memory; some systems of this batch are unsolved");
  else if (rc != HYDIST_OK) hyd::set_last_error("hydist_gtsv_batched: a CUDA call failed");
  return rc;
}

// ---- FP32 solve refined once with an FP64 residual -------------------------
extern "C" int hydist_gtsv_batched_refine(const double* dl, const double* d, const double* du,
                                          const double* b, double* x, const int32_t* offsets,
                                          const int32_t* lengths, int32_t nsys, int32_t algo,
                                          void* stream) {
  if (!dl || !d || !du || !b || !x || !offsets || !lengths || nsys < 0) {
    hyd::set_last_error("hydist_gtsv_batched_refine: null pointer or negative count");
    return HYDIST_ERR_ARG;
  }
  if (algo < HYDIST_GTSV_AUTO || algo > HYDIST_GTSV_PIVOT) {
    hyd::set_last_error("hydist_gtsv_batched_refine: unknown algo");
    return HYDIST_ERR_ARG;
  }
  if (nsys == 0) return HYDIST_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return HYDIST_ERR_CUDA;
  // the packed extent, for the FP32 copies (a device reduction of off+len)
  size_t rows = 0;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    DevInfo* D = dev_info(dev);
    if (!D) return HYDIST_ERR_ARG;
    int rc = ensure_scratch(D->scr, 0, (size_t)nsys);
    if (rc != HYDIST_OK) return rc;
    if (cudaMemsetAsync(D->scr.counts, 0, (GT_NB + 2) * sizeof(int), st) != cudaSuccess)
      return HYDIST_ERR_CUDA;
    hyd::k_gt_classify<<<(nsys + 255) / 256, 256, 0, st>>>(offsets, lengths, nsys, D->scr.lists,
                                                           D->scr.counts);
    int counts[GT_NB + 2];
    if (cudaMemcpyAsync(counts, D->scr.counts, sizeof(counts), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return HYDIST_ERR_CUDA;
    if (counts[GT_NB + 1]) {
      hyd::set_last_error("hydist_gtsv_batched_refine: a system has a negative offset");
      return HYDIST_ERR_ARG;
    }
    rows = (size_t)counts[GT_NB];
    // each FP32 array starts 16-byte aligned (the CTA solvers stage rows
    // with bulk copies)
    const size_t need = (rows + 3) / 4 * 4 * 5 * sizeof(float);
    if (D->scr.f32_bytes < need) {
      if (D->scr.f32) cudaFree(D->scr.f32);
      D->scr.f32 = nullptr;
      D->scr.f32_bytes = 0;
      if (cudaMalloc(&D->scr.f32, need + 256) != cudaSuccess) return HYDIST_ERR_OOM;
      D->scr.f32_bytes = need;
    }
  }
  if (rows == 0) return HYDIST_OK;
  float* f = nullptr;
  int nsm = 1;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    f = dev_info(dev)->scr.f32;
    nsm = dev_info(dev)->nsm;
  }
  const size_t ld = (rows + 3) / 4 * 4;
  float *fl = f, *fd = f + ld, *fu = f + 2 * ld, *fb = f + 3 * ld, *fx = f + 4 * ld;
  hyd::k_gt_to_f32<<<4 * nsm, 256, 0, st>>>(dl, d, du, b, f, rows, ld);
  int rc = hydist_gtsv_batched(fl, fd, fu, fb, fx, offsets, lengths, nsys, 1, algo, stream);
  if (rc != HYDIST_OK) return rc;
  // x = x32, r = b - A x32 in FP64, into fb as the correction's right-hand side
  hyd::k_gt_residual<<<nsys, 128, 0, st>>>(dl, d, du, b, fx, x, fb, offsets, lengths, nsys);
  rc = hydist_gtsv_batched(fl, fd, fu, fb, fx, offsets, lengths, nsys, 1, algo, stream);
  if (rc != HYDIST_OK) return rc;
  hyd::k_gt_correct<<<nsys, 128, 0, st>>>(x, fx, offsets, lengths, nsys);
  if (cudaGetLastError() != cudaSuccess) {
    hyd::set_last_error("hydist_gtsv_batched_refine: a kernel launch failed");
    return HYDIST_ERR_CUDA;
  }
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
  thomas_system(dl + o, d + o, du + o, b + o, x + o, w + o, n);
}

}  // namespace hyd

namespace {
constexpr int kNoallocDevices = 64;
std::mutex g_noalloc_mu;
// scratch address per device, with the context it was looked up in: a
// device reset gives the device a new context (and the array a new
// address), which the next call notices and looks the address up again
struct NoallocSlot {
  void* ctx = nullptr;
  void* ptr = nullptr;
};
NoallocSlot g_noalloc[kNoallocDevices];

// the driver's cuCtxGetCurrent through the runtime's entry-point query (the
// library links only the runtime); null if the driver does not offer it
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
  static const CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (CtxGetCurrentFn)p;
  }();
  return fn;
}

void* current_ctx() {
  void* c = nullptr;
  const CtxGetCurrentFn f = ctx_get_current();
  if (!f || f(&c) != 0) return nullptr;
  return c;
}
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
    NoallocSlot& slot = g_noalloc[dev];
    void* ctx = current_ctx();
    if (!slot.ptr || !ctx || ctx != slot.ctx) {
      // set-up on this device (and again after a reset of its context)
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, hyd::g_noalloc_w);
      if (e != cudaSuccess || !p) {
        hyd::set_last_error("hydist_gtsv_batched_noalloc: cudaGetSymbolAddress failed");
        return HYDIST_ERR_CUDA;
      }
      slot.ptr = p;
      slot.ctx = current_ctx();  // current now that the runtime has set the device up
    }
    w = slot.ptr;
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
