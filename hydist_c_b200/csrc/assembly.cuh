// assembly.cuh -- per-cell coefficients of the hydraulic ADI systems.
//
// pre_x / pre_y restate _uzSolver_calculate_preindex / _vzSolver_calculate_
// preindex (UVZSolver_multithread.cpp:210-278, 142-208), abcd restates
// _calculate_abcd (:280-342), line_sys and row_of the row layout of
// _calculate_matrix_coeff with bienrandau / bienlongdau (:110-139, 345-470).
// Expression order follows the reference.
#pragma once

#include "common.cuh"

namespace hyd {

// Per-cell coefficients of the preindex step.
struct Pre {
  double f1, f2, f3, f5, a2, c2, d2;
};

// _uzSolver_calculate_preindex (UVZSolver_multithread.cpp:210-278).
__device__ __forceinline__ Pre pre_x(const State& S, const Coef& c, int i, int j) {
  const int w = S.W;
  const double* u = S.u;
  const double* v = S.v;
  const double* Hm = S.Hmoi;
  Pre P;
  double p = 0.0, q = 0.0;
  const double vtb =
      (v[i * w + j - 1] + v[i * w + j] + v[(i + 1) * w + j - 1] + v[(i + 1) * w + j]) * 0.25;
  const double uu = u[i * w + j], VI = S.visco[i * w + j], Hu = S.Htdu[i * w + j];
  const double dT = c.dT;
  P.f1 = c.dTchia2dX * uu + VI * dT / c.dXbp;
  P.f2 = -(2 + S.Kx1[i * w + j] * dT * sqrt(uu * uu + vtb * vtb) / Hu + (2 * dT * VI) / c.dXbp);
  P.f3 = dT * VI / c.dXbp - c.dTchia2dX * uu;
  if (Hm[i * w + j - 1] <= c.H_TINH) {
    if (vtb < 0) {
      p = vtb * (-3 * uu + 4 * u[i * w + j + 1] - u[i * w + j + 2]) / c.dY2;
      q = (uu - 2 * u[i * w + j + 1] + u[i * w + j + 2]) / c.dYbp;
    }
  } else {
    if (Hm[i * w + j + 1] <= c.H_TINH) {
      if ((Hm[i * w + j - 2] > c.H_TINH) && (vtb > 0)) {
        p = vtb * (3 * uu - 4 * u[i * w + j - 1] + u[i * w + j - 2]) / c.dY2;
        q = (uu - 2 * u[i * w + j - 1] + u[i * w + j - 2]) / c.dYbp;
      }
    } else {
      p = vtb * (u[i * w + j + 1] - u[i * w + j - 1]) / c.dY2;
      q = (u[i * w + j + 1] - 2 * uu + u[i * w + j - 1]) / c.dYbp;
    }
  }
  P.f5 = -2 * uu + dT * p - dT * c.CORIOLIS_FORCE * vtb - dT * VI * q -
         dT * (c.Windx - S.Tsxw[i * w + j]) / Hu;
  P.c2 = c.dTchia2dX * Hu;
  P.a2 = -c.dTchia2dX * S.Htdu[(i - 1) * w + j];
  P.d2 = S.z[i * w + j] -
         c.dTchia2dY * (S.Htdv[i * w + j] * v[i * w + j] - S.Htdv[i * w + j - 1] * v[i * w + j - 1]);
  return P;
}

// _vzSolver_calculate_preindex (UVZSolver_multithread.cpp:142-208).
__device__ __forceinline__ Pre pre_y(const State& S, const Coef& c, int i, int j) {
  const int w = S.W;
  const double* u = S.u;
  const double* v = S.v;
  const double* Hm = S.Hmoi;
  Pre P;
  double p = 0.0, q = 0.0;
  const double utb =
      (u[(i - 1) * w + j] + u[i * w + j] + u[(i - 1) * w + j + 1] + u[i * w + j + 1]) * 0.25;
  const double vv = v[i * w + j], VI = S.visco[i * w + j], Hv = S.Htdv[i * w + j];
  const double dT = c.dT;
  P.f1 = c.dTchia2dY * vv + VI * dT / c.dYbp;
  P.f2 = -(2 + S.Ky1[i * w + j] * dT * sqrt(vv * vv + utb * utb) / Hv + (2 * dT * VI) / c.dYbp);
  P.f3 = dT * VI / c.dYbp - c.dTchia2dY * vv;
  if (Hm[(i - 1) * w + j] <= c.H_TINH) {
    if (utb < 0) {
      q = utb * (-3 * vv + 4 * v[(i + 1) * w + j] - v[(i + 2) * w + j]) / c.dX2;
      p = (vv - 2 * v[(i + 1) * w + j] + v[(i + 2) * w + j]) / c.dXbp;
    }
  } else {
    if (Hm[(i + 1) * w + j] <= c.H_TINH) {
      if ((Hm[(i - 2) * w + j] > c.H_TINH) && (utb > 0)) {
        q = utb * (3 * vv - 4 * v[(i - 1) * w + j] + v[(i - 2) * w + j]) / c.dX2;
        p = (vv - 2 * v[(i - 1) * w + j] + v[(i - 2) * w + j]) / c.dXbp;
      }
    } else {
      q = utb * (v[(i + 1) * w + j] - v[(i - 1) * w + j]) / c.dX2;
      p = (v[(i + 1) * w + j] - 2 * vv + v[(i - 1) * w + j]) / c.dXbp;
    }
  }
  P.f5 = -2 * vv + dT * q + dT * c.CORIOLIS_FORCE * utb - dT * VI * p -
         dT * (c.Windy - S.Tsyw[i * w + j]) / Hv;
  P.c2 = c.dTchia2dY * Hv;
  P.a2 = -c.dTchia2dY * S.Htdv[i * w + j - 1];
  P.d2 = S.z[i * w + j] -
         c.dTchia2dX * (S.Htdu[i * w + j] * u[i * w + j] - S.Htdu[(i - 1) * w + j] * u[(i - 1) * w + j]);
  return P;
}

struct Mom {
  double a1, b1, c1, d1;
};

// _calculate_abcd (UVZSolver_multithread.cpp:280-342) at position k of a
// segment [first, last]; P = cell k, Pn = cell k+1 (read only when used).
__device__ __forceinline__ Mom abcd(const Pre& P, const Pre& Pn, int k, int first, int last,
                                    double f4, bool br1, bool br2) {
  Mom m;
  if (last - 1 > first) {
    if (br1 && k == first) {
      m.a1 = f4;
      m.b1 = P.f2 - (P.f3 * Pn.a2 / Pn.c2);
      m.c1 = -f4 - (P.f3 / Pn.c2);
      m.d1 = P.f5 - (P.f3 * Pn.d2 / Pn.c2);
    } else if (br2 && k == last - 1) {
      m.a1 = f4 - P.f1 / P.a2;
      m.b1 = P.f2 - (P.f1 * P.c2 / P.a2);
      m.c1 = -f4;
      m.d1 = P.f5 - (P.f1 * P.d2 / P.a2);
    } else {
      m.a1 = f4 - P.f1 / P.a2;
      m.c1 = -f4 - (P.f3 / Pn.c2);
      m.b1 = P.f2 - (P.f1 * P.c2 / P.a2) - (P.f3 * Pn.a2 / Pn.c2);
      m.d1 = P.f5 - (P.f1 * P.d2 / P.a2) - (P.f3 * Pn.d2 / Pn.c2);
    }
  } else {
    m.a1 = f4;
    m.b1 = P.f2;
    m.d1 = P.f5;
    m.c1 = -f4;
  }
  return m;
}

// Streaming Thomas forward pass (tridiag, UVZSolver_multithread.cpp:19-43):
// rows arrive in order k = 0..sn; Ap/Bp go to scratch.
struct ThomasFwd {
  double ap, bp, xs;
  int sn;
  double* Ap;
  double* Bp;
  int ld;
  __device__ __forceinline__ void row(int k, int r, double A, double B, double Cc, double D) {
    if (k == 0) {
      if (sn == 0) {
        xs = D / B;
        return;
      }
      ap = -Cc / B;
      bp = D / B;
      Ap[(size_t)r * ld] = ap;
      Bp[(size_t)r * ld] = bp;
    } else if (k < sn) {
      const double ep = A * ap + B;
      ap = -Cc / ep;
      bp = (D - (A * bp)) / ep;
      Ap[(size_t)r * ld] = ap;
      Bp[(size_t)r * ld] = bp;
    } else {
      xs = (D - (A * bp)) / (B + (A * ap));
    }
  }
};

// Layout of one line's solve: which of the reference's assembly variants
// applies (UVZSolver_multithread.cpp:377-465) and where the system ends.
struct LineSys {
  bool ran;      // continuity row first (solid or discharge first end)
  bool qfirst;   // discharge at the first end
  int last_kind; // 0 solid, 1 discharge, 2 water level
  int off, sn;
};

__device__ __forceinline__ LineSys line_sys(int first, int last, bool br1, bool br2, bool q1,
                                            bool q2, int dkfr) {
  LineSys L;
  L.off = 2 * first;
  int sn = 2 * (last - first);
  if (br1) {
    L.ran = true;
    L.qfirst = false;
    if (!br2) {
      if (q2 && last == dkfr) {
        L.last_kind = 1;
      } else {
        sn--;
        L.last_kind = 2;
      }
    } else {
      L.last_kind = 0;
    }
  } else {
    const bool isBienran = (q1 && first == 2);
    L.ran = isBienran;
    L.qfirst = isBienran;
    if (!br2) {
      if (q1 && last == dkfr) {  // the first end's flag (UVZSolver_multithread.cpp:438)
        if (!isBienran) sn--;
        L.last_kind = 1;
      } else {
        sn--;
        if (!isBienran) sn -= 1;
        L.last_kind = 2;
      }
    } else {
      if (!isBienran) sn--;
      L.last_kind = 0;
    }
  }
  L.sn = sn;
  return L;
}

// Coefficients of absolute row r of a line's system (see line_sys).
__device__ __forceinline__ void row_of(const LineSys& L, int r, const Pre& Pi, const Mom& Mi,
                                       const Pre& Pi1, double& A, double& B, double& Cc,
                                       double& D) {
  const bool even = (r & 1) == 0;
  if (L.ran == even) {  // continuity row of cell i (ran) / cell i+1 (lon)
    const Pre& P = L.ran ? Pi : Pi1;
    A = P.a2;
    B = 1;
    Cc = P.c2;
    D = P.d2;
  } else {  // momentum row of cell i
    A = Mi.a1;
    B = Mi.b1;
    Cc = Mi.c1;
    D = Mi.d1;
  }
}

}  // namespace hyd
