// sediment_cell.cuh -- per-cell coefficients of the concentration sweeps.
//
// The formulas keep the structure of the reference's (sources below); the
// powers with constant exponents are products and square roots
// ((1-FS)^4, Pd^2.5, Tx^1.5), pow(Dxr, -0.3) is a constant of Coef, and the
// divisions by constants and by H_moi are multiplications by reciprocals.
// Each changes a result by a few roundings at most.
#pragma once

#include "common.cuh"

namespace hyd {

// source_chs (sediment_transport.cpp:11-38)
template <class R>
__device__ __forceinline__ R source_chs(const CoefT<R>& c, R wsm, R Zf, R fs, R fw, R vth,
                                        R h_moi) {
  R toee = c.Toe;
  R S = 0;
  const R tob = c.ro * fw * (vth * vth);
  if (h_moi > c.ghtoe) toee = toee * (1 + c.hstoe * ((h_moi - c.ghtoe)));
  if (tob > toee) {
    S = c.Mb_ros * (tob - toee) / toee;
  } else if (tob < c.Tod) {
    const R Pd = 1 - tob * c.r_Tod;
    const R beta = 1 + (Zf / (R(1.25) + R(4.75) * (Pd * Pd * sqrt(Pd))));
    const R Cb = beta * fs;
    S = -wsm * Cb * Pd;
  }
  return S;
}

// source_nchs (sediment_transport.cpp:41-49)
template <class R>
__device__ __forceinline__ R source_nchs(const CoefT<R>& c, R wsm, R Zf, R Uf, R r_hmoi, R fs) {
  const R gamac = R(0.434) + R(5.975) * Zf + R(2.888) * Zf * Zf;
  const R Tx = fmax(R(0), (Uf * Uf - c.Ufr * c.Ufr) * c.r_Ufr2);
  const R Cac = R(0.015) * c.dm * (Tx * sqrt(Tx)) * c.Dxr_m03 * (R(20) * r_hmoi);
  return wsm * (Cac - gamac * fs);
}

// Calculate_Qb (sediment_transport.cpp:352-434) at cell (i, j) of rows
// 2..N, columns 2..M, read as intended where the code cannot be meant
// literally: the flux where the speed is not zero (:385 divides by the VTH
// it tests to be zero), Toee starting from the coefficient Toe (:359), both
// components in the corner copies (:410-419). vth, kh, Hm, fw are the cell's
// speed, mask, H_moi and Fw; tu, tu_up = t_u(i, j), t_u(i-1, j); tv,
// tv_left = t_v(i, j), t_v(i, j-1). The margins and corners copy the
// nearest interior value (:402-431).
template <class R>
__device__ __forceinline__ void qb_cell(const StateT<R>& S, const CoefT<R>& c, int i, int j,
                                        R vth, int kh, R Hm, R fw, R tu, R tu_up, R tv,
                                        R tv_left) {
  const int w = S.W, pos = i * w + j, N = S.N, M = S.M;
  R qx = 0, qy = 0;
  if (vth != 0 && kh == 0) {
    R Toee = c.Toe, Tx = 0;
    const R Tob = c.ro * fw * (vth * vth);
    if (Hm > c.ghtoe) Toee = c.Toe * (1 + c.hstoe * ((Hm - c.ghtoe)));
    if (Tob > Toee) Tx = Tob / Toee - 1;
    const R base = c.qb_k * pow(Tx, R(2.1)) * c.Dxr_m03;
    qx = base * (tu + tu_up) * R(0.5) / vth;
    qy = base * (tv + tv_left) * R(0.5) / vth;
  }
  R* Qbx = S.Qbx;
  R* Qby = S.Qby;
  Qbx[pos] = qx;
  Qby[pos] = qy;
  if (i == 2) {
    Qbx[pos - w] = qx;
    Qby[pos - w] = qy;
  }
  if (i == N) {
    Qbx[pos + w] = qx;
    Qby[pos + w] = qy;
  }
  if (j == 2) {
    Qbx[pos - 1] = qx;
    Qby[pos - 1] = qy;
    if (i == 2) {
      Qbx[1 * w + 1] = qx;
      Qby[1 * w + 1] = qy;
    }
    if (i == N) {
      Qbx[(N + 1) * w + 1] = qx;
      Qby[(N + 1) * w + 1] = qy;
    }
  }
  if (j == M) {
    Qbx[pos + 1] = qx;
    Qby[pos + 1] = qy;
    if (i == 2) {
      Qbx[1 * w + M + 1] = qx;
      Qby[1 * w + M + 1] = qy;
    }
    if (i == N) {
      Qbx[(N + 1) * w + M + 1] = qx;
      Qby[(N + 1) * w + M + 1] = qy;
    }
  }
}

// One cell's row of a concentration sweep: xdir = _FSj (:204-313), else
// _FSi (:51-164). The along-line values are passed in by the caller, which
// carries them from cell to cell: vel_c / hk_c are the sweep-direction
// velocity and Htd*K product of this cell (x: tu, Htdu*Kx at pos; y: tv,
// Htdv*Ky at pos), vel_p / hk_p those of the cell before it (pos-W in x,
// pos-1 in y).
template <class R>
__device__ __forceinline__ void fs_cell(const StateT<R>& S, const CoefT<R>& c, bool xdir, int i,
                                        int j, R vel_c, R hk_c, R vel_p, R hk_p, double tt,
                                        double s_start, R& A, R& B, R& Cc, R& D) {
  const int w = S.W, pos = i * w + j;
  const R* Hm = S.Hmoi;
  const R* FS = S.FS;
  const R H_TINH = c.H_TINH;
  const R Hc = Hm[pos], fs = FS[pos], vth = S.VTH[pos];
  const R rH = R(1) / Hc;
  const R cc = 18 * log(12 * Hc / c.Ks);
  const R Uf = c.sqrt_g * fabs(vth) / cc;
  const R om = 1 - fs, om2 = om * om;
  const R wsm = c.wss * (om2 * om2);
  R Zf = 0, Sx;
  if (fs > R(0.00001)) Zf = wsm / (R(0.4) * (Uf + 2 * wsm));
  // the i-sweep evaluates gamav before Zf (:247), the j-sweep after it (:109)
  const R gamav = xdir ? R(0.98) : R(0.98) - R(0.198) * Zf + R(0.032) * Zf * Zf;
  if (S.ketdinh)
    Sx = source_chs(c, wsm, Zf, fs, S.Fw[pos], vth, Hc);
  else
    Sx = source_nchs(c, wsm, Zf, Uf, rH, fs);
  if (tt < s_start) Sx = 0;
  // along-line terms
  const R r_d2 = xdir ? c.r_dX2 : c.r_dY2;      // 1 / (2 d)
  const R r_dd = (xdir ? c.r_dXbp : c.r_dYbp) * rH;  // 1 / (H_moi d^2)
  const R adv = gamav * R(0.5) * (vel_c + vel_p) * r_d2;
  A = -adv - hk_p * r_dd;
  Cc = adv - hk_c * r_dd;
  B = c.HaiChiadT + (hk_c + hk_p) * r_dd;
  // cross-line terms
  const int s = xdir ? 1 : w;  // stride across the sweep
  const R* vx = xdir ? S.tv : S.tu;
  const R* hx = xdir ? S.Htdv : S.Htdu;
  const R* kx = xdir ? S.Ky : S.Kx;
  const R hm1 = Hm[pos - s], hp1 = Hm[pos + s], hm2 = Hm[pos - 2 * s], hp2 = Hm[pos + 2 * s];
  const R fm = FS[pos - s], fp = FS[pos + s];
  const R vxc = vx[pos], vxm = vx[pos - s];  // before the tests that use them
  R p = 0, q = 0;
  if ((hm1 > H_TINH) && (hp2 > H_TINH)) p = (fp - fs);
  if ((hm2 > H_TINH) && (hp1 > H_TINH)) q = (fs - fm);
  p = (rH * (xdir ? c.r_dYbp : c.r_dXbp)) * (hx[pos] * kx[pos] * p - hx[pos - s] * kx[pos - s] * q);
  if ((hm2 > H_TINH) && (hp2 > H_TINH)) {
    q = (fp - fm) * (xdir ? c.r_dY2 : c.r_dX2);
    q = (vxc + vxm) * R(0.5) * q * gamav;
  } else {
    q = 0;
  }
  D = fs * c.HaiChiadT - q + p + Sx * rH;
}

}  // namespace hyd
