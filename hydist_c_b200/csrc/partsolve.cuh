// partsolve.cuh -- partition-method solve of one tridiagonal system held in
// shared memory by a warp, and the reduced-system work space of the CTA
// solver (tridiag.cu).
//
// Rows r = 0..n-1: A_r x_{r-1} + B_r x_r + C_r x_{r+1} = D_r, A_0 = C_{n-1} = 0.
// The system is cut into chunks of S unknowns (the last chunk takes the
// remainder, so every chunk has at least 2); chunk k belongs to thread k:
//   pass A  forward elimination of the chunk's interior keeping the spike of
//           the previous chunk's separator: x_r = y'_r + v'_r x_L - c'_r x_{r+1},
//           (c', y', v') written over the rows in place; the chunk's last
//           unknown is its separator. The first interior row in terms of both
//           neighbouring separators is accumulated on the way;
//   reduce  the separators form a tridiagonal system of one unknown per
//           chunk, solved by parallel cyclic reduction (shared memory for a
//           CTA, shuffles for a warp);
//   pass C  back substitution, x written over D.
// Shared-memory index of row q is q + q/S (one pad slot per chunk), so the
// chunks a warp walks in step fall on different banks.
#pragma once

#include <cuda_runtime.h>

namespace hyd {

__host__ __device__ inline int part_idx(int q, int S) { return q + q / S; }

// part_idx of q = t0, t0 + dt, t0 + 2 dt, ... without a division per step:
// carries the quotient and remainder of q / S.
struct PartStrideIdx {
  int q, qd, qr, dd, dr, S;
  __device__ PartStrideIdx(int t0, int dt, int S_) : q(t0), qd(t0 / S_), qr(t0 % S_), dd(dt / S_), dr(dt % S_), S(S_) {}
  __device__ int idx() const { return q + qd; }
  __device__ void next(int dt) {
    q += dt;
    qd += dd;
    qr += dr;
    if (qr >= S) {
      qr -= S;
      ++qd;
    }
  }
};

struct PartGeom {
  int S;       // unknowns per chunk (>= 2)
  int nchunk;  // chunks, <= threads
  int stride;  // elements per row array
};

// Upper bound of part_geom(n, threads).stride over all lengths <= nmax
// (the stride itself is not monotonic in n): sizes shared memory for a band.
__host__ __device__ inline int part_stride_bound(int nmax, int threads) {
  return nmax + (nmax / 2 < threads ? nmax / 2 : threads) + 2;
}

__host__ __device__ inline PartGeom part_geom(int n, int threads) {
  PartGeom g;
  g.S = (n + threads - 1) / threads;
  if (g.S < 2) g.S = 2;
  g.nchunk = n / g.S;
  if (g.nchunk < 1) g.nchunk = 1;
  g.stride = n + n / g.S + 2;
  return g;
}

// Chunk k's forward elimination. Writes (c', y', v') over (C, D, A) of the
// interior rows and returns the separator row and the chunk's couplings:
// tri = (yF, vF, wF, yL, vL, wL): first interior unknown = yF + vF x_L + wF x_sep,
// last interior unknown = yL + vL x_L + wL x_sep.
// Index of row q0 + s of chunk k (q0 = k*S): k*(S+1) + s, one more once s
// reaches S (only the last chunk is that long).
__device__ __forceinline__ int part_chunk_idx(int k, int S, int s) {
  return k * (S + 1) + s + (s >= S ? 1 : 0);
}

template <class T>
__device__ __forceinline__ void part_forward(T* rA, T* rB, T* rC, T* rD, int q0, int nu, int S,
                                             T sep[4], T tri[6]) {
  T cp = 0, yp = 0, vp = 0;
  T Pk = 1, fy = 0, fv = 0;
  const int k = q0 / S;
  for (int s = 0; s < nu; ++s) {
    const int o = part_chunk_idx(k, S, s);
    const T A = rA[o], B = rB[o], C = rC[o], D = rD[o];
    if (s == nu - 1) {
      sep[0] = A;
      sep[1] = B;
      sep[2] = C;
      sep[3] = D;
    } else {
      if (s == 0) {
        const T m = T(1) / B;
        cp = C * m;
        yp = D * m;
        vp = -A * m;
      } else {
        const T m = T(1) / (B - A * cp);
        yp = (D - A * yp) * m;
        vp = -A * vp * m;
        cp = C * m;
      }
      rC[o] = cp;
      rD[o] = yp;
      rA[o] = vp;
      fy += Pk * yp;
      fv += Pk * vp;
      Pk *= -cp;
    }
  }
  tri[0] = fy;
  tri[1] = fv;
  tri[2] = Pk;
  tri[3] = yp;
  tri[4] = vp;
  tri[5] = -cp;
}

template <class T>
__device__ __forceinline__ void part_back(T* rA, T* rC, T* rD, int q0, int nu, int S, T xl, T xr) {
  const int k = q0 / S;
  rD[part_chunk_idx(k, S, nu - 1)] = xr;
  T xn = xr;
  for (int t = nu - 2; t >= 0; --t) {
    const int o = part_chunk_idx(k, S, t);
    const T x = rD[o] + rA[o] * xl - rC[o] * xn;
    rD[o] = x;
    xn = x;
  }
}

// Reduced-system work space of a CTA of NT threads.
template <class T, int NT>
struct PartCtaShared {
  T tri[3][NT];  // yF vF wF of each chunk (read by the previous chunk)
  T red[4][NT];
  T xsep[NT];
};

// Warp-wide solve (all 32 lanes call it; the rows are in the warp's slice of
// shared memory). The reduced system is solved with shuffles.
template <class T>
__device__ void part_solve_warp(T* rA, T* rB, T* rC, T* rD, const PartGeom& g, int n, int lane) {
  const unsigned full = 0xffffffffu;
  const int k = lane, P = g.nchunk, S = g.S;
  const int q0 = k * S;
  const int nu = k < P ? ((k == P - 1) ? n - q0 : S) : 0;
  T sep[4] = {0, 1, 0, 0}, tri[6] = {0, 0, 1, 0, 0, 0};
  if (k < P) part_forward(rA, rB, rC, rD, q0, nu, S, sep, tri);
  const T yF = __shfl_down_sync(full, tri[0], 1);
  const T vF = __shfl_down_sync(full, tri[1], 1);
  const T wF = __shfl_down_sync(full, tri[2], 1);
  T ra = 0, rb = 1, rc = 0, rd = 0;
  if (k < P) {
    const bool nx = k + 1 < P;
    ra = sep[0] * tri[4];
    rb = sep[1] + sep[0] * tri[5] + sep[2] * (nx ? vF : T(0));
    rc = sep[2] * (nx ? wF : T(0));
    rd = sep[3] - sep[0] * tri[3] - sep[2] * (nx ? yF : T(0));
  }
  for (int st = 1; st < P; st <<= 1) {
    T am = __shfl_up_sync(full, ra, st), bm = __shfl_up_sync(full, rb, st);
    T cm = __shfl_up_sync(full, rc, st), dm = __shfl_up_sync(full, rd, st);
    T an = __shfl_down_sync(full, ra, st), bn = __shfl_down_sync(full, rb, st);
    T cn = __shfl_down_sync(full, rc, st), dn = __shfl_down_sync(full, rd, st);
    if (!(k < P && k - st >= 0)) {
      am = 0;
      bm = 1;
      cm = 0;
      dm = 0;
    }
    if (!(k + st < P)) {
      an = 0;
      bn = 1;
      cn = 0;
      dn = 0;
    }
    const T k1 = ra / bm, k2 = rc / bn;
    const T na = -am * k1, nc = -cn * k2;
    const T nb = rb - cm * k1 - an * k2;
    const T nd = rd - dm * k1 - dn * k2;
    ra = na;
    rb = nb;
    rc = nc;
    rd = nd;
  }
  const T xs = rd / rb;
  const T xl = __shfl_up_sync(full, xs, 1);
  if (k < P) part_back(rA, rC, rD, q0, nu, S, k > 0 ? xl : T(0), xs);
  __syncwarp();
}

}  // namespace hyd
