// uvz_compat.cu -- the reference's UVZSolver kernels (UVZSolver_multithread.h:
// 6-55) with their C++ signatures, for programs that drive the ADI
// half-steps themselves, as the reference's engine.cpp does, and swap only
// the solver objects.
//
// Each kernel keeps the reference's launch contract -- which cell or line a
// thread takes from the launch shape and the index arguments, and which it
// skips -- and writes the same intermediate arrays of Array_Pointers in the
// same layout: f1..f5, a2, c2, d2 and a1..d1 per line with width N+2 (x
// sweep, line j) or M+2 (y sweep, line i); AA..DD and x per line with width
// 2N+1 / 2M+1; SN per segment (line*20 + segment). The caller's remaining
// kernels (Normalize, update_buffer, the commits, the concentration sweeps,
// which also call tridiagSolver) read them unchanged. The cell arithmetic is
// this library's (assembly.cuh, explicit.cuh), so results agree with the
// reference's to rounding.
//
// Where several of the reference's threads write one location with
// different values and the launch order decides, one thread writes the value
// the reference's own runs produce: the first and last rows of a segment's
// system are the end conditions, and the end velocity recovered from
// continuity reads the neighbour written in the same launch (the new value).
// Positions whose values no system reads (a1..d1 at a segment's last cell,
// rows past a system's last row) are not written.
//
// Every kernel is compiled for blocks of up to 1024 threads, the largest the
// reference launches (its 2D launches take min(1024, M+3) threads).
//
// This is the kernel-level drop-in, not the fast path: Hydraulic_Calculation
// (compat.cu) and hydist_step run a half-step without these arrays.
#include <cuda_runtime.h>

#include "../../include/hydist_gtsv_device.cuh"
#include "../../include/hydist_uvz_compat.h"
#include "assembly.cuh"
#include "common.cuh"
#include "explicit.cuh"

namespace {

using hyd::Coef;
using hyd::Mom;
using hyd::Pre;
using hyd::SEG;
using hyd::State;

// The coefficients the cell arithmetic reads, from the caller's
// Constant_Coeffs (whose derived members Load_coeffs has set).
__device__ Coef coef_of(const Constant_Coeffs* k) {
  Coef c{};
  c.dX = k->dX;
  c.dY = k->dY;
  c.dT = k->dT;
  c.dXbp = k->dXbp;
  c.dYbp = k->dYbp;
  c.dX2 = k->dX2;
  c.dY2 = k->dY2;
  c.dTchia2dX = k->dTchia2dX;
  c.dTchia2dY = k->dTchia2dY;
  c.HaiChiadT = k->HaiChiadT;
  c.NANGDAY = k->NANGDAY;
  c.H_TINH = k->H_TINH;
  c.CORIOLIS_FORCE = k->CORIOLIS_FORCE;
  c.g = k->g;
  c.Windx = k->Windx;
  c.Windy = k->Windy;
  c.r_dX = 1.0 / c.dX;
  c.r_dY = 1.0 / c.dY;
  c.r_dX2 = 1.0 / c.dX2;
  c.r_dY2 = 1.0 / c.dY2;
  c.r_dXbp = 1.0 / c.dXbp;
  c.r_dYbp = 1.0 / c.dYbp;
  c.dT_dXbp = c.dT / c.dXbp;
  c.dT_dYbp = c.dT / c.dYbp;
  return c;
}

// A State view of the caller's arrays (the fields the cell arithmetic reads).
__device__ State state_of(const Argument_Pointers* a) {
  State S{};
  S.M = a->M;
  S.N = a->N;
  S.W = a->M + 3;
  S.H = a->N + 3;
  S.h = a->h;
  S.u = a->u;
  S.v = a->v;
  S.z = a->z;
  S.tz = a->t_z;
  S.tu = a->t_u;
  S.tv = a->t_v;
  S.Hmoi = a->H_moi;
  S.Htdu = a->Htdu;
  S.Htdv = a->Htdv;
  S.visco = a->VISCOIDX;
  S.Kx1 = a->Kx1;
  S.Ky1 = a->Ky1;
  S.Tsxw = a->Tsxw;
  S.Tsyw = a->Tsyw;
  S.daui = a->daui;
  S.cuoii = a->cuoii;
  S.moci = a->moci;
  S.dauj = a->dauj;
  S.cuoij = a->cuoij;
  S.mocj = a->mocj;
  return S;
}

// The wet segment of a line that holds a position, with its solid-end flags.
struct Loc {
  int k, first, last;
  bool br1, br2;
};

// locate_segment_u (support_funcs.cpp:832-858): column j, row i.
__device__ bool locate_u(const Argument_Pointers* a, double NANGDAY, int i, int j, Loc& L) {
  const int n = a->mocj[j], w = a->M + 3, N = a->N;
  for (int k = 0; k < n; ++k) {
    const int f = a->dauj[j * SEG + k], l = a->cuoij[j * SEG + k];
    if (f <= i && i <= l) {
      L.k = k;
      L.first = f;
      L.last = l;
      L.br1 = (f > 2) || (f == 2 && (a->h[1 * w + j] + a->h[1 * w + j - 1]) * 0.5 == NANGDAY);
      L.br2 = (l < N) || (l == N && (a->h[N * w + j] + a->h[N * w + j - 1]) * 0.5 == NANGDAY);
      return true;
    }
  }
  return false;
}

// locate_segment_v (support_funcs.cpp:810-830): row i, column j.
__device__ bool locate_v(const Argument_Pointers* a, double NANGDAY, int i, int j, Loc& L) {
  const int n = a->moci[i], w = a->M + 3, M = a->M;
  for (int k = 0; k < n; ++k) {
    const int f = a->daui[i * SEG + k], l = a->cuoii[i * SEG + k];
    if (f <= j && j <= l) {
      L.k = k;
      L.first = f;
      L.last = l;
      L.br1 = (f > 2) || (f == 2 && (a->h[i * w + f - 1] + a->h[(i - 1) * w + f - 1]) * 0.5 == NANGDAY);
      L.br2 = (l < M) || (l == M && (a->h[i * w + l] + a->h[(i - 1) * w + l]) * 0.5 == NANGDAY);
      return true;
    }
  }
  return false;
}

__device__ void put_pre(Array_Pointers* arr, int o, const Pre& P) {
  arr->f1[o] = P.f1;
  arr->f2[o] = P.f2;
  arr->f3[o] = P.f3;
  arr->f5[o] = P.f5;
  arr->a2[o] = P.a2;
  arr->c2[o] = P.c2;
  arr->d2[o] = P.d2;
}

__device__ Pre get_pre(const Array_Pointers* arr, int o) {
  return Pre{arr->f1[o], arr->f2[o], arr->f3[o], arr->f5[o], arr->a2[o], arr->c2[o], arr->d2[o]};
}

// _calculate_abcd (UVZSolver_multithread.cpp:280-342) at position k of a
// segment of the line whose support arrays start at `base`.
__device__ void abcd_at(Array_Pointers* arr, int base, int k, const Loc& L, double f4) {
  Mom m;
  if (L.last - 1 > L.first) {
    if (k == L.last) return;  // read by no system
    const Pre P = get_pre(arr, base + k), Pn = get_pre(arr, base + k + 1);
    m = hyd::abcd(P, Pn, k, L.first, L.last, f4, L.br1, L.br2);
  } else {
    // one momentum row: every thread of the reference's segment writes it
    if (k != L.first) return;
    const Pre P = get_pre(arr, base + k);
    m = hyd::abcd(P, P, k, L.first, L.last, f4, L.br1, L.br2);
  }
  arr->a1[base + k] = m.a1;
  arr->b1[base + k] = m.b1;
  arr->c1[base + k] = m.c1;
  arr->d1[base + k] = m.d1;
}

// _calculate_matrix_coeff with bienrandau / bienlongdau (UVZSolver_
// multithread.cpp:110-139, 345-470): the rows of position k of a segment on
// line `line`; the position at the segment's first and last cells also
// writes the end conditions and the system size SN.
__device__ void assemble_at(Array_Pointers* arr, int line, int k, int sw, int tw, const Loc& L,
                            double ub_first, double ub_last, double TZ_r, double TZ_l, bool q1,
                            bool q2, int dkfr) {
  const int first = L.first, last = L.last, off = 2 * first;
  const hyd::LineSys Ls = hyd::line_sys(first, last, L.br1, L.br2, q1, q2, dkfr);
  const int rlast = off + Ls.sn;  // the system's last row
  double* AA = arr->AA + (size_t)line * tw;
  double* BB = arr->BB + (size_t)line * tw;
  double* CC = arr->CC + (size_t)line * tw;
  double* DD = arr->DD + (size_t)line * tw;
  const double* a1 = arr->a1 + (size_t)line * sw;
  const double* b1 = arr->b1 + (size_t)line * sw;
  const double* c1 = arr->c1 + (size_t)line * sw;
  const double* d1 = arr->d1 + (size_t)line * sw;
  const double* a2 = arr->a2 + (size_t)line * sw;
  const double* c2 = arr->c2 + (size_t)line * sw;
  const double* d2 = arr->d2 + (size_t)line * sw;
  // rows 2k and 2k+1: continuity of k then momentum of k (the first end a
  // continuity row), or momentum of k then continuity of k+1
  for (int e = 0; e < 2; ++e) {
    const int r = 2 * k + e;
    if (r >= rlast) break;
    const bool cont = Ls.ran ? (e == 0) : (e == 1);
    const int p = Ls.ran ? k : (e == 0 ? k : k + 1);
    if (cont) {
      AA[r] = a2[p];
      BB[r] = 1;
      CC[r] = c2[p];
      DD[r] = d2[p];
    } else {
      AA[r] = a1[k];
      BB[r] = b1[k];
      CC[r] = c1[k];
      DD[r] = d1[k];
    }
  }
  if (k == first && rlast > off) {
    // the first end (a system of one row takes the last end's form below)
    if (Ls.ran) {
      DD[off] = Ls.qfirst ? d2[first] - a2[first] * ub_first : d2[first];
    } else {
      BB[off] = b1[first];
      CC[off] = c1[first];
      DD[off] = d1[first] - a1[first] * TZ_l;
    }
  }
  if (k == last) {
    if (rlast == off && !Ls.ran) CC[off] = c1[first];
    if (Ls.last_kind == 1) {
      AA[rlast] = a2[last];
      BB[rlast] = 1;
      DD[rlast] = d2[last] - c2[last] * ub_last;
    } else if (Ls.last_kind == 2) {
      AA[rlast] = a1[last - 1];
      BB[rlast] = b1[last - 1];
      DD[rlast] = d1[last - 1] - c1[last - 1] * TZ_r;
    } else {
      AA[rlast] = a2[last];
      BB[rlast] = 1;
      DD[rlast] = d2[last];
    }
    arr->SN[line * SEG + L.k] = Ls.sn;
  }
}

// tridiag (UVZSolver_multithread.cpp:19-43): Thomas on rows 0..sn with the
// caller's scratch Ap, Bp, ep.
__device__ void thomas(int sn, const double* A, const double* B, const double* C, const double* D,
                       double* x, double* Ap, double* Bp, double* ep) {
  if (sn < 0) return;  // a degenerate one-cell segment: nothing to solve
  if (sn == 0) {
    x[0] = D[0] / B[0];
    return;
  }
  Ap[0] = -C[0] / B[0];
  Bp[0] = D[0] / B[0];
  for (int i = 1; i < sn; ++i) {
    ep[i] = A[i] * Ap[i - 1] + B[i];
    Ap[i] = -C[i] / ep[i];
    Bp[i] = (D[i] - A[i] * Bp[i - 1]) / ep[i];
  }
  x[sn] = (D[sn] - A[sn] * Bp[sn - 1]) / (B[sn] + A[sn] * Ap[sn - 1]);
  for (int i = sn - 1; i >= 0; --i) x[i] = Bp[i] + Ap[i] * x[i + 1];
}

// The value the extraction writes to the velocity at position p of a
// segment's system (p in [first, last)), as _uz/_vzSolver_extract_solution
// do: the continuity-first layout puts it at 2p+1, the momentum-first one at
// 2p (and at 2 first for the first cell).
__device__ double vel_of(const double* x, int p, int first, bool ran) {
  return ran ? x[2 * p + 1] : x[2 * p];
}

// _uzSolver_extract_solution / _vzSolver_extract_solution (UVZSolver_
// multithread.cpp:547-603, 472-544) at position k of a segment. z and vel
// point at the line's first cell (stride s), so position p is z[p * s].
__device__ void extract_at(const double* x, const double* a2, const double* c2, const double* d2,
                           double* z, double* vel, int s, int k, int sn, const Loc& L, bool q1,
                           bool q2, double ub_first, double ub_last, int dkfr) {
  const int first = L.first, last = L.last;
  const bool ran = L.br1 || (q1 && first == 2);
  if (k < last) {
    if (ran) {
      z[k * s] = x[2 * k];
      vel[k * s] = x[2 * k + 1];
      if (k == first) vel[(first - 1) * s] = L.br1 ? 0.0 : ub_first;
    } else if (k == first) {
      vel[first * s] = x[2 * first];
      vel[(first - 1) * s] = (d2[first] - z[first * s] - c2[first] * vel[first * s]) / a2[first];
    } else {
      z[k * s] = x[2 * k - 1];
      vel[k * s] = x[2 * k];
    }
    return;
  }
  if (L.br2) {
    vel[last * s] = 0;
    z[last * s] = x[2 * first + sn];
  } else if (q2 && last == dkfr) {
    vel[last * s] = ub_last;
    z[last * s] = x[2 * first + sn];
  } else {
    // continuity at the last cell with the neighbour's velocity of this
    // launch (written by position last-1 when it lies in the segment)
    const double vn = last - 1 >= first ? vel_of(x, last - 1, first, ran) : vel[(last - 1) * s];
    vel[last * s] = (d2[last] - a2[last] * vn - z[last * s]) / c2[last];
  }
}

// the calling thread's index in its block and the block's size
__device__ int flat_tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ int flat_nthreads() { return blockDim.x * blockDim.y * blockDim.z; }

}  // namespace

// ------------------------------------------------------------- y sweep (VZ)

// VZSolver_calculate_preindex (UVZSolver_multithread.cpp:798-808).
__global__ void __launch_bounds__(1024) VZSolver_calculate_preindex(int startidx, int endidx, Argument_Pointers* arg,
                                            Array_Pointers* arr, Constant_Coeffs* coeffs) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (i > endidx || j > arg->M) return;
  Loc L;
  if (!locate_v(arg, coeffs->NANGDAY, i, j, L)) return;
  const State S = state_of(arg);
  const Coef c = coef_of(coeffs);
  put_pre(arr, i * (arg->M + 2) + j, hyd::pre_y(S, c, i, j));
}

// VZSolver_calculate_abcd (UVZSolver_multithread.cpp:813-829).
__global__ void __launch_bounds__(1024) VZSolver_calculate_abcd(int startidx, int endidx, Argument_Pointers* arg,
                                        Array_Pointers* arr, Constant_Coeffs* coeffs) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (i > endidx || j > arg->M) return;
  Loc L;
  if (!locate_v(arg, coeffs->NANGDAY, i, j, L)) return;
  abcd_at(arr, i * (arg->M + 2), j, L, 2 * coeffs->g * coeffs->dTchia2dY);
}

// VZSolver_calculate_matrix_coeff (UVZSolver_multithread.cpp:831-843). SN
// is written at row*20 + segment for rows up to N: the caller's SN must hold
// 20*(N+1) ints.
__global__ void __launch_bounds__(1024) VZSolver_calculate_matrix_coeff(int startidx, int endidx, double NANGDAY,
                                                Argument_Pointers* arg, Array_Pointers* arr) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int M = arg->M;
  if (i > endidx || j > M) return;
  Loc L;
  if (!locate_v(arg, NANGDAY, i, j, L)) return;
  const int w = M + 3;
  assemble_at(arr, i, j, M + 2, 2 * M + 1, L, arg->vbd[i], arg->vbt[i], arg->t_z[i * w + L.last],
              arg->t_z[i * w + L.first], arg->bienQ[1] != 0, arg->bienQ[0] != 0, M);
}

// VZSolver_extract_solution (UVZSolver_multithread.cpp:845-859); like the
// reference it tests the column against endidx.
__global__ void __launch_bounds__(1024) VZSolver_extract_solution(int startidx, int endidx, double NANGDAY,
                                          Argument_Pointers* arg, Array_Pointers* arr) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (j > endidx || i > arg->N) return;
  Loc L;
  if (!locate_v(arg, NANGDAY, i, j, L)) return;
  const int M = arg->M, w = M + 3;
  const int sn = arr->SN[i * SEG + L.k];
  extract_at(arr->x + (size_t)i * (2 * M + 1), arr->a2 + (size_t)i * (M + 2),
             arr->c2 + (size_t)i * (M + 2), arr->d2 + (size_t)i * (M + 2), arg->t_z + (size_t)i * w,
             arg->t_v + (size_t)i * w, 1, j, sn, L, arg->bienQ[1] != 0, arg->bienQ[0] != 0,
             arg->vbd[i], arg->vbt[i], M);
}

// solveV (UVZSolver_multithread.cpp:961-978) with vSolver (:607-663).
__global__ void __launch_bounds__(1024) solveV(double t, int startidx, int endidx, Argument_Pointers* arg,
                       Constant_Coeffs* coeffs) {
  (void)t;
  const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  if (i > endidx || j > arg->M) return;
  Loc L;
  if (!locate_v(arg, coeffs->NANGDAY, i, j, L)) return;
  if (L.first >= L.last || j >= L.last) return;
  const State S = state_of(arg);
  const Coef c = coef_of(coeffs);
  const int g = i * S.W + j;
  arg->t_v[g] = hyd::v_new(hyd::v_ops(S, static_cast<const double*>(arg->t_u), g), c);
}

// update_margin_elem_V (UVZSolver_multithread.cpp:1018-1060): row
// blockIdx.y * blockDim.y + threadIdx.y + startidx (the reference's other
// threads of the block repeat the same writes).
__global__ void __launch_bounds__(1024) update_margin_elem_V(int startidx, int endidx, double NANGDAY,
                                     Argument_Pointers* arg) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  if (i > endidx || threadIdx.x != 0 || threadIdx.z != 0) return;
  hyd::margin_v(state_of(arg), NANGDAY, i);
}

// ------------------------------------------------------------- x sweep (UZ)

// UZSolver_calculate_preindex (UVZSolver_multithread.cpp:876-891).
__global__ void __launch_bounds__(1024) UZSolver_calculate_preindex(int startidx, int endidx, Argument_Pointers* arg,
                                            Array_Pointers* arr, Constant_Coeffs* coeffs) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + startidx;
  if (j > endidx || i > arg->N) return;
  Loc L;
  if (!locate_u(arg, coeffs->NANGDAY, i, j, L)) return;
  const State S = state_of(arg);
  const Coef c = coef_of(coeffs);
  put_pre(arr, j * (arg->N + 2) + i, hyd::pre_x(S, c, i, j));
}

// UZSolver_calculate_abcd (UVZSolver_multithread.cpp:894-913).
__global__ void __launch_bounds__(1024) UZSolver_calculate_abcd(int startidx, int endidx, Argument_Pointers* arg,
                                        Array_Pointers* arr, Constant_Coeffs* coeffs) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + startidx;
  if (j > endidx || i > arg->N) return;
  Loc L;
  if (!locate_u(arg, coeffs->NANGDAY, i, j, L)) return;
  abcd_at(arr, j * (arg->N + 2), i, L, 2 * coeffs->g * coeffs->dTchia2dX);
}

// UZSolver_calculate_matrix_coeff (UVZSolver_multithread.cpp:916-933).
__global__ void __launch_bounds__(1024) UZSolver_calculate_matrix_coeff(int startidx, int endidx, double NANGDAY,
                                                Argument_Pointers* arg, Array_Pointers* arr) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + startidx;
  const int N = arg->N;
  if (j > endidx || i > N) return;
  Loc L;
  if (!locate_u(arg, NANGDAY, i, j, L)) return;
  const int w = arg->M + 3;
  assemble_at(arr, j, i, N + 2, 2 * N + 1, L, arg->ubt[j], arg->ubp[j], arg->t_z[L.last * w + j],
              arg->t_z[L.first * w + j], arg->bienQ[2] != 0, arg->bienQ[3] != 0, N);
}

// UZSolver_extract_solution (UVZSolver_multithread.cpp:861-873).
__global__ void __launch_bounds__(1024) UZSolver_extract_solution(int startidx, int endidx, double NANGDAY,
                                          Argument_Pointers* arg, Array_Pointers* arr) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + startidx;
  if (j > endidx || i > arg->N) return;
  Loc L;
  if (!locate_u(arg, NANGDAY, i, j, L)) return;
  const int N = arg->N, w = arg->M + 3;
  const int sn = arr->SN[j * SEG + L.k];
  extract_at(arr->x + (size_t)j * (2 * N + 1), arr->a2 + (size_t)j * (N + 2),
             arr->c2 + (size_t)j * (N + 2), arr->d2 + (size_t)j * (N + 2), arg->t_z + j,
             arg->t_u + j, w, i, sn, L, arg->bienQ[2] != 0, arg->bienQ[3] != 0, arg->ubt[j],
             arg->ubp[j], N);
}

// solveU (UVZSolver_multithread.cpp:938-959) with uSolver (:724-795).
__global__ void __launch_bounds__(1024) solveU(double t, int startidx, int endidx, Argument_Pointers* arg,
                       Constant_Coeffs* coeffs) {
  (void)t;
  const int i = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int j = blockIdx.x * blockDim.x + threadIdx.x + startidx;
  if (i > arg->N || j > endidx) return;
  Loc L;
  if (!locate_u(arg, coeffs->NANGDAY, i, j, L)) return;
  if (L.first > L.last || i < L.first - 1 || i >= L.last) return;
  const State S = state_of(arg);
  const Coef c = coef_of(coeffs);
  const int ij = i * S.W + j;
  arg->t_u[ij] = hyd::u_new(hyd::u_ops(S, static_cast<const double*>(arg->t_v), ij), c);
}

// update_margin_elem_U (UVZSolver_multithread.cpp:980-1016): column
// blockIdx.y * blockDim.y + threadIdx.y + startidx.
__global__ void __launch_bounds__(1024) update_margin_elem_U(int startidx, int endidx, double NANGDAY,
                                     Argument_Pointers* arg) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y + startidx;
  if (j > endidx || threadIdx.x != 0 || threadIdx.z != 0) return;
  hyd::margin_u(state_of(arg), NANGDAY, j);
}

// ---------------------------------------------------- tridiagonal solvers

// tridiagSolver (UVZSolver_multithread.cpp:78-109): the segments of line
// blockIdx.y + startidx, the system of segment s at line*width +
// first*jumpstep + jumpstep%2 with SN[line*20 + s] + 1 rows. The reference's
// threads of a block all repeat the same solve; here they take the
// segments in turn.
__global__ void __launch_bounds__(1024) tridiagSolver(bool print, bool isU, int startidx, int endidx, int jumpstep,
                              int tridiag_coeff_width, Argument_Pointers* arg, Array_Pointers* arr) {
  (void)print;
  const int i = blockIdx.y + startidx;
  if (i > endidx) return;
  const int n = isU ? arg->mocj[i] : arg->moci[i];
  const int* dau = isU ? arg->dauj : arg->daui;
  for (int s = flat_tid(); s < n; s += flat_nthreads()) {
    const int first = dau[i * SEG + s];
    const size_t pos = (size_t)i * tridiag_coeff_width + first * jumpstep + jumpstep % 2;
    thomas(arr->SN[i * SEG + s], arr->AA + pos, arr->BB + pos, arr->CC + pos, arr->DD + pos,
           arr->x + pos, arr->Ap + pos, arr->Bp + pos, arr->ep + pos);
  }
}

// tridiagSolver_v2 (UVZSolver_multithread.cpp:47-75): line threadIdx.x +
// startidx, each segment through gtsv_spike_partial_diag_pivot_v1
// (hydist_gtsv_device.cuh) with m = SN as the reference passes it.
__global__ void __launch_bounds__(1024) tridiagSolver_v2(bool print, bool isU, int startidx, int endidx, int jumpstep,
                                 int tridiag_coeff_width, Argument_Pointers* arg,
                                 Array_Pointers* arr) {
  (void)print;
  const int i = threadIdx.x + startidx;
  if (i > endidx) return;
  const int n = isU ? arg->mocj[i] : arg->moci[i];
  const int* dau = isU ? arg->dauj : arg->daui;
  for (int s = 0; s < n; ++s) {
    const int first = dau[i * SEG + s];
    const size_t pos = (size_t)i * tridiag_coeff_width + first * jumpstep + jumpstep % 2;
    gtsv_spike_partial_diag_pivot_v1(arr->AA + pos, arr->BB + pos, arr->CC + pos, arr->DD + pos,
                                     arr->x + pos, arr->SN[i * SEG + s]);
  }
}
