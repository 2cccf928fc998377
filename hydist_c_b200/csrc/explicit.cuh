// explicit.cuh -- per-cell explicit momentum updates and per-line segment-end
// velocities, shared by the fused half-steps (hydro.cu) and the reference's
// kernel-level entry points (uvz_compat.cu).
//
// v_new restates vSolver (UVZSolver_multithread.cpp:607-663), u_new uSolver
// (:724-795, where dX and Windx are read from dY and Windy as the reference
// does, :731, :734); margin_v / margin_u restate update_margin_elem_V / _U
// (:1018-1060, :980-1016). Operands are gathered into a struct first so that
// a caller can issue every load before anything that decides whether the
// cell is updated (one round of memory latency).
#pragma once

#include "common.cuh"

namespace hyd {

// Operands of vSolver at cell g; tu is t_u after its smoothing.
template <class R>
struct VOps {
  R u00, u01, u10, u11, t00, t01, t10, t11;
  R vv, vl, vr, vm1, vm2, vp1, vp2, hm1, hm2, hp1;
  R Hv, Ky1, vis, tsy, dz;
};

template <class R>
__device__ __forceinline__ VOps<R> v_ops(const StateT<R>& S, const R* tu, int g) {
  const int off = S.W;
  const R* u = S.u;
  const R* v = S.v;
  const R* Hm = S.Hmoi;
  VOps<R> o;
  o.u00 = u[g - off];
  o.u01 = u[g];
  o.u10 = u[g - off + 1];
  o.u11 = u[g + 1];
  o.t00 = tu[g - off];
  o.t01 = tu[g];
  o.t10 = tu[g - off + 1];
  o.t11 = tu[g + 1];
  o.vv = v[g];
  o.vl = v[g - 1];
  o.vr = v[g + 1];
  o.vm1 = v[g - off];
  o.vm2 = v[g - 2 * off];
  o.vp1 = v[g + off];
  o.vp2 = v[g + 2 * off];
  o.hm1 = Hm[g - off];
  o.hm2 = Hm[g - 2 * off];
  o.hp1 = Hm[g + off];
  o.Hv = S.Htdv[g];
  o.Ky1 = S.Ky1[g];
  o.vis = S.visco[g];
  o.tsy = S.Tsyw[g];
  o.dz = R(S.z[g + 1] - S.z[g]);  // the level difference in FP64 first
  return o;
}

template <class R>
__device__ __forceinline__ R v_new(const VOps<R>& o, const CoefT<R>& c) {
  R p, q = 0, tmp = 0;
  const R vv = o.vv;
  const R utb = (o.u00 + o.u01 + o.u10 + o.u11) * R(0.25);
  const R t_utb = (o.t00 + o.t01 + o.t10 + o.t11) * R(0.25);
  const R rHv = R(1) / o.Hv;
  p = (o.vr - o.vl) * c.r_dY2;
  p = c.HaiChiadT + p + o.Ky1 * sqrt(utb * utb + vv * vv) * rHv;
  if (o.hm1 <= c.H_TINH) {
    if (utb < 0) {
      q = t_utb * (-3 * vv + 4 * o.vp1 - o.vp2) * c.r_dX2;
      tmp = (vv - 2 * o.vp1 + o.vp2) * c.r_dXbp;
    }
  } else {
    if (o.hp1 <= c.H_TINH) {
      if ((o.hm2 > c.H_TINH) && (utb > 0)) {
        q = t_utb * (3 * vv - 4 * o.vm1 + o.vm2) * c.r_dX2;
        tmp = (vv - 2 * o.vm1 + o.vm2) * c.r_dXbp;
      }
    } else {
      q = t_utb * (o.vp1 - o.vm1) * c.r_dX2;
      tmp = (o.vp1 - 2 * vv + o.vm1) * c.r_dXbp;
    }
  }
  q = c.HaiChiadT * vv - q - c.CORIOLIS_FORCE * t_utb;
  q = (q - c.g * o.dz * c.r_dY + o.vis * (tmp + (o.vr - 2 * vv + o.vl) * c.r_dYbp)) +
      (c.Windy - o.tsy) * rHv;
  return q / p;
}

// Operands of uSolver at cell ij (rows 1..N, columns 2..M: all in bounds);
// tv is t_v after its smoothing.
template <class R>
struct UOps {
  R v00, v01, v10, v11, t00, t01, t10, t11;
  R uu, ud, uup, ul1, ul2, ur1, ur2, hl1, hl2, hr1;
  R Hu, Kx1, vis, tsx, dz;
};

template <class R>
__device__ __forceinline__ UOps<R> u_ops(const StateT<R>& S, const R* tv, int ij) {
  const int off = S.W, i1j = ij + off;
  const R* u = S.u;
  const R* v = S.v;
  const R* Hm = S.Hmoi;
  UOps<R> o;
  o.v00 = v[ij - 1];
  o.v01 = v[ij];
  o.v10 = v[i1j - 1];
  o.v11 = v[i1j];
  o.t00 = tv[ij - 1];
  o.t01 = tv[ij];
  o.t10 = tv[i1j - 1];
  o.t11 = tv[i1j];
  o.uu = u[ij];
  o.ud = u[i1j];
  o.uup = u[ij - off];
  o.ul1 = u[ij - 1];
  o.ul2 = u[ij - 2];
  o.ur1 = u[ij + 1];
  o.ur2 = u[ij + 2];
  o.hl1 = Hm[ij - 1];
  o.hl2 = Hm[ij - 2];
  o.hr1 = Hm[ij + 1];
  o.Hu = S.Htdu[ij];
  o.Kx1 = S.Kx1[ij];
  o.vis = S.visco[ij];
  o.tsx = S.Tsxw[ij];
  o.dz = R(S.z[i1j] - S.z[ij]);  // the level difference in FP64 first
  return o;
}

template <class R>
__device__ __forceinline__ R u_new(const UOps<R>& o, const CoefT<R>& c) {
  const R Windx = c.Windy;
  // dX is read from dY: 1/(2dX) = r_dY2, 1/dX^2 = r_dYbp, 1/dX = r_dY
  R p, q = 0, tmp = 0;
  const R uu = o.uu;
  const R vtb = (o.v00 + o.v01 + o.v10 + o.v11) * R(0.25);
  const R t_vtb = (o.t00 + o.t01 + o.t10 + o.t11) * R(0.25);
  const R rHu = R(1) / o.Hu;
  p = (o.ud - o.uup) * c.r_dY2;
  p = (c.HaiChiadT + p + o.Kx1 * sqrt(vtb * vtb + uu * uu) * rHu);
  if (o.hl1 <= c.H_TINH) {
    if (vtb < 0) {
      q = t_vtb * (-3 * uu + 4 * o.ur1 - o.ur2) * c.r_dY2;
      tmp = (uu - 2 * o.ur1 + o.ur2) * c.r_dYbp;
    }
  } else {
    if (o.hr1 <= c.H_TINH) {
      if ((o.hl2 > c.H_TINH) && (vtb > 0)) {
        q = t_vtb * (3 * uu - 4 * o.ul1 + o.ul2) * c.r_dY2;
        tmp = (uu - 2 * o.ul1 + o.ul2) * c.r_dYbp;
      }
    } else {
      q = t_vtb * (o.ur1 - o.ul1) * c.r_dY2;
      tmp = (o.ur1 - 2 * uu + o.ul1) * c.r_dYbp;
    }
  }
  q = c.HaiChiadT * uu - q + c.CORIOLIS_FORCE * t_vtb;
  q = (q - c.g * o.dz * c.r_dY + o.vis * (tmp + (o.ud - 2 * uu + o.uup) * c.r_dYbp)) +
      (Windx - o.tsx) * rHu;
  return q / p;
}

// Segment-end velocities of row i (update_margin_elem_V): zero at a solid
// end, linear extrapolation at an open one.
template <class R>
__device__ __forceinline__ void margin_v(const StateT<R>& S, double NANGDAY, int i) {
  const int w = S.W, M = S.M;
  R* tv = S.tv;
  for (int k = 0; k < S.moci[i]; ++k) {
    const int first = S.daui[i * SEG + k], last = S.cuoii[i * SEG + k];
    const bool br1 = (first > 2) || ((first == 2) && (fabs((S.h[i * w + first - 1] + S.h[(i - 1) * w + first - 1]) * 0.5 - NANGDAY) < 1e-16));
    const bool br2 = (last < M) || ((last == M) && (fabs((S.h[i * w + last] + S.h[(i - 1) * w + last]) * 0.5 - NANGDAY) < 1e-16));
    if (br1) tv[i * w + first - 1] = 0;
    else tv[i * w + first - 1] = 2 * tv[i * w + first] - tv[i * w + first + 1];
    if (br2) tv[i * w + last] = 0;
    else tv[i * w + last] = 2 * tv[i * w + last - 1] - tv[i * w + last - 2];
  }
}

// Segment-end velocities of column j (update_margin_elem_U).
template <class R>
__device__ __forceinline__ void margin_u(const StateT<R>& S, double NANGDAY, int j) {
  const int w = S.W, N = S.N;
  R* tu = S.tu;
  for (int k = 0; k < S.mocj[j]; ++k) {
    const int first = S.dauj[j * SEG + k], last = S.cuoij[j * SEG + k];
    const bool br1 = (first > 2) || ((first == 2) && (fabs((S.h[1 * w + j] + S.h[1 * w + j - 1]) * 0.5 - NANGDAY) < 1e-16));
    const bool br2 = (last < N) || ((last == N) && (fabs((S.h[N * w + j] + S.h[N * w + j - 1]) * 0.5 - NANGDAY) < 1e-16));
    if (br1) tu[(first - 1) * w + j] = 0;
    else tu[(first - 1) * w + j] = 2 * tu[first * w + j] - tu[(first + 1) * w + j];
    if (br2) tu[last * w + j] = 0;
    else tu[last * w + j] = 2 * tu[(last - 1) * w + j] - tu[(last - 2) * w + j];
  }
}

}  // namespace hyd
