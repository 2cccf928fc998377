// assembly.cuh -- per-cell coefficients of the hydraulic ADI systems.
//
// pre_x / pre_y restate _uzSolver_calculate_preindex / _vzSolver_calculate_
// preindex (UVZSolver_multithread.cpp:210-278, 142-208), abcd restates
// _calculate_abcd (:280-342), line_sys the row layout of
// _calculate_matrix_coeff with bienrandau / bienlongdau (:110-139, 345-470).
//
// The formulas keep the reference's structure; divisions by constants are
// multiplications by precomputed reciprocals (Coef::r_*), and each cell
// takes one reciprocal of Htdu (or Htdv), of a2 and of the next cell's c2
// instead of the reference's repeated divisions. This changes results by a
// rounding at most per operation, and keeps exact zeros exact.
#pragma once

#include "common.cuh"

namespace hyd {

// Per-cell coefficients of the preindex step, in the step's type R.
template <class R>
struct PreT {
  R f1, f2, f3, f5, a2, c2, d2;
};
using Pre = PreT<double>;

// _uzSolver_calculate_preindex (UVZSolver_multithread.cpp:210-278).
template <class R>
__device__ __forceinline__ PreT<R> pre_x(const StateT<R>& S, const CoefT<R>& c, int i, int j) {
  const int w = S.W;
  const int g = i * w + j;
  const R* u = S.u;
  const R* v = S.v;
  const R* Hm = S.Hmoi;
  PreT<R> P;
  R p = 0, q = 0;
  const R vtb = (v[g - 1] + v[g] + v[g + w - 1] + v[g + w]) * R(0.25);
  const R uu = u[g], VI = S.visco[g], Hu = S.Htdu[g];
  const R dT = c.dT;
  const R rH = R(1) / Hu;
  const R visc = VI * c.dT_dXbp;
  P.f1 = c.dTchia2dX * uu + visc;
  P.f2 = -(2 + S.Kx1[g] * dT * sqrt(uu * uu + vtb * vtb) * rH + 2 * visc);
  P.f3 = visc - c.dTchia2dX * uu;
  if (Hm[g - 1] <= c.H_TINH) {
    if (vtb < 0) {
      p = vtb * (-3 * uu + 4 * u[g + 1] - u[g + 2]) * c.r_dY2;
      q = (uu - 2 * u[g + 1] + u[g + 2]) * c.r_dYbp;
    }
  } else {
    if (Hm[g + 1] <= c.H_TINH) {
      if ((Hm[g - 2] > c.H_TINH) && (vtb > 0)) {
        p = vtb * (3 * uu - 4 * u[g - 1] + u[g - 2]) * c.r_dY2;
        q = (uu - 2 * u[g - 1] + u[g - 2]) * c.r_dYbp;
      }
    } else {
      p = vtb * (u[g + 1] - u[g - 1]) * c.r_dY2;
      q = (u[g + 1] - 2 * uu + u[g - 1]) * c.r_dYbp;
    }
  }
  P.f5 = -2 * uu + dT * p - dT * c.CORIOLIS_FORCE * vtb - dT * VI * q -
         dT * (c.Windx - S.Tsxw[g]) * rH;
  P.c2 = c.dTchia2dX * Hu;
  P.a2 = -c.dTchia2dX * S.Htdu[g - w];
  P.d2 = R(S.z[g]) - c.dTchia2dY * (S.Htdv[g] * v[g] - S.Htdv[g - 1] * v[g - 1]);
  return P;
}

// _vzSolver_calculate_preindex (UVZSolver_multithread.cpp:142-208).
template <class R>
__device__ __forceinline__ PreT<R> pre_y(const StateT<R>& S, const CoefT<R>& c, int i, int j) {
  const int w = S.W;
  const int g = i * w + j;
  const R* u = S.u;
  const R* v = S.v;
  const R* Hm = S.Hmoi;
  PreT<R> P;
  R p = 0, q = 0;
  const R utb = (u[g - w] + u[g] + u[g - w + 1] + u[g + 1]) * R(0.25);
  const R vv = v[g], VI = S.visco[g], Hv = S.Htdv[g];
  const R dT = c.dT;
  // the cross-line stencil (rows i-2..i+2, inside the array for rows 2..N)
  // loaded before the upwind tests choose from it
  const R vm1 = v[g - w], vm2 = v[g - 2 * w], vp1 = v[g + w], vp2 = v[g + 2 * w];
  const R hm1 = Hm[g - w], hp1 = Hm[g + w], hm2 = Hm[g - 2 * w];
  const R rH = R(1) / Hv;
  const R visc = VI * c.dT_dYbp;
  P.f1 = c.dTchia2dY * vv + visc;
  P.f2 = -(2 + S.Ky1[g] * dT * sqrt(vv * vv + utb * utb) * rH + 2 * visc);
  P.f3 = visc - c.dTchia2dY * vv;
  if (hm1 <= c.H_TINH) {
    if (utb < 0) {
      q = utb * (-3 * vv + 4 * vp1 - vp2) * c.r_dX2;
      p = (vv - 2 * vp1 + vp2) * c.r_dXbp;
    }
  } else {
    if (hp1 <= c.H_TINH) {
      if ((hm2 > c.H_TINH) && (utb > 0)) {
        q = utb * (3 * vv - 4 * vm1 + vm2) * c.r_dX2;
        p = (vv - 2 * vm1 + vm2) * c.r_dXbp;
      }
    } else {
      q = utb * (vp1 - vm1) * c.r_dX2;
      p = (vp1 - 2 * vv + vm1) * c.r_dXbp;
    }
  }
  P.f5 = -2 * vv + dT * q + dT * c.CORIOLIS_FORCE * utb - dT * VI * p -
         dT * (c.Windy - S.Tsyw[g]) * rH;
  P.c2 = c.dTchia2dY * Hv;
  P.a2 = -c.dTchia2dY * S.Htdv[g - 1];
  P.d2 = R(S.z[g]) - c.dTchia2dX * (S.Htdu[g] * u[g] - S.Htdu[g - w] * u[g - w]);
  return P;
}

template <class R>
struct MomT {
  R a1, b1, c1, d1;
};
using Mom = MomT<double>;

// _calculate_abcd (UVZSolver_multithread.cpp:280-342) at position k of a
// segment [first, last]; P = cell k, Pn = cell k+1 (read only when used).
template <class R>
__device__ __forceinline__ MomT<R> abcd(const PreT<R>& P, const PreT<R>& Pn, int k, int first,
                                       int last, R f4, bool br1, bool br2) {
  MomT<R> m;
  if (last - 1 > first) {
    if (br1 && k == first) {
      const R rc = P.f3 / Pn.c2;
      m.a1 = f4;
      m.b1 = P.f2 - rc * Pn.a2;
      m.c1 = -f4 - rc;
      m.d1 = P.f5 - rc * Pn.d2;
    } else if (br2 && k == last - 1) {
      const R ra = P.f1 / P.a2;
      m.a1 = f4 - ra;
      m.b1 = P.f2 - ra * P.c2;
      m.c1 = -f4;
      m.d1 = P.f5 - ra * P.d2;
    } else {
      const R ra = P.f1 / P.a2, rc = P.f3 / Pn.c2;
      m.a1 = f4 - ra;
      m.c1 = -f4 - rc;
      m.b1 = P.f2 - ra * P.c2 - rc * Pn.a2;
      m.d1 = P.f5 - ra * P.d2 - rc * Pn.d2;
    }
  } else {
    m.a1 = f4;
    m.b1 = P.f2;
    m.d1 = P.f5;
    m.c1 = -f4;
  }
  return m;
}

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

}  // namespace hyd
