// sediment_cell.cuh -- per-cell coefficients of the concentration sweeps.
#pragma once

#include "common.cuh"

namespace hyd {

// source_chs (sediment_transport.cpp:11-38)
__device__ __forceinline__ double source_chs(const Coef& c, double wsm, double Zf, double fs,
                                             double fw, double vth, double h_moi) {
  double toee = c.Toe;
  const double todd = c.Tod;
  double S = 0;
  const double tob = c.ro * fw * (vth * vth);
  if (h_moi > c.ghtoe) toee = toee * (1 + c.hstoe * ((h_moi - c.ghtoe)));
  if (tob > toee) {
    S = c.Mbochat / c.ros * (tob - toee) / toee;
  } else if (tob < todd) {
    const double Pd = 1 - (tob / todd);
    const double beta = 1 + (Zf / (1.25 + 4.75 * pow(Pd, 2.5)));
    const double Cb = beta * fs;
    S = -wsm * Cb * Pd;
  }
  return S;
}

// source_nchs (sediment_transport.cpp:41-49)
__device__ __forceinline__ double source_nchs(const Coef& c, double wsm, double Zf, double Uf,
                                              double h_moi, double fs) {
  const double gamac = 0.434 + 5.975 * Zf + 2.888 * Zf * Zf;
  const double Tx = fmax(0.0, (Uf * Uf - c.Ufr * c.Ufr) / (c.Ufr * c.Ufr));
  const double Cac = 0.015 * c.dm * pow(Tx, 1.5) * pow(c.Dxr, (-0.3)) / (0.05 * h_moi);
  return wsm * (Cac - gamac * fs);
}

// One cell's row of a concentration sweep: xdir = _FSj (:204-313), else
// _FSi (:51-164).
__device__ __forceinline__ void fs_cell(const State& S, const Coef& c, bool xdir, int i, int j,
                                        double tt, double s_start, double& A, double& B,
                                        double& Cc, double& D) {
  const int w = S.W, pos = i * w + j;
  const double* Hm = S.Hmoi;
  const double* FS = S.FS;
  const double dX = c.dX, dY = c.dY, dT = c.dT, H_TINH = c.H_TINH;
  const double cc = 18 * log(12 * Hm[pos] / c.Ks);
  const double Uf = sqrt(c.g) * fabs(S.VTH[pos]) / cc;
  const double wsm = c.wss * pow((1 - FS[pos]), 4.0);
  double Zf = 0, Sx;
  double gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
  if (FS[pos] > 0.00001) Zf = wsm / (0.4 * (Uf + 2 * wsm));
  if (S.ketdinh)
    Sx = source_chs(c, wsm, Zf, FS[pos], S.Fw[pos], S.VTH[pos], Hm[pos]);
  else
    Sx = source_nchs(c, wsm, Zf, Uf, Hm[pos], FS[pos]);
  if (tt < s_start) Sx = 0;
  double p = 0, q = 0;
  if (xdir) {
    A = -gamav * 0.5 * (S.tu[pos] + S.tu[pos - w]) / (dX * 2) -
        S.Htdu[pos - w] * S.Kx[pos - w] / (Hm[pos] * (dX * dX));
    Cc = gamav * 0.5 * (S.tu[pos] + S.tu[pos - w]) / (dX * 2) -
         S.Htdu[pos] * S.Kx[pos] / (Hm[pos] * (dX * dX));
    B = 2.0 / dT + (S.Htdu[pos] * S.Kx[pos] + S.Htdu[pos - w] * S.Kx[pos - w]) / (Hm[pos] * (dX * dX));
    if ((Hm[pos - 1] > H_TINH) && (Hm[pos + 2] > H_TINH)) p = (FS[pos + 1] - FS[pos]);
    if ((Hm[pos - 2] > H_TINH) && (Hm[pos + 1] > H_TINH)) q = (FS[pos] - FS[pos - 1]);
    p = (1 / (Hm[pos] * (dY * dY))) * (S.Htdv[pos] * S.Ky[pos] * p - S.Htdv[pos - 1] * S.Ky[pos - 1] * q);
    if ((Hm[pos - 2] > H_TINH) && (Hm[pos + 2] > H_TINH)) {
      q = (FS[pos + 1] - FS[pos - 1]) / (dY * 2);
      q = (S.tv[pos] + S.tv[pos - 1]) * 0.5 * q * gamav;
    } else {
      q = 0;
    }
  } else {
    gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;
    A = -gamav * 0.5 * (S.tv[pos - 1] + S.tv[pos]) / (dY * 2) -
        S.Htdv[pos - 1] * S.Ky[pos - 1] / (Hm[pos] * (dY * dY));
    Cc = gamav * 0.5 * (S.tv[pos - 1] + S.tv[pos]) / (dY * 2) -
         S.Htdv[pos] * S.Ky[pos] / (Hm[pos] * (dY * dY));
    B = 2.0 / dT + (S.Htdv[pos] * S.Ky[pos] + S.Htdv[pos - 1] * S.Ky[pos - 1]) / (Hm[pos] * (dY * dY));
    if ((Hm[pos + 2 * w] > H_TINH) && (Hm[pos - w] > H_TINH)) p = (FS[pos + w] - FS[pos]);
    if (Hm[pos - 2 * w] > H_TINH && Hm[pos + w] > H_TINH) q = (FS[pos] - FS[pos - w]);
    p = (1 / (Hm[pos] * (dX * dX))) * (S.Htdu[pos] * S.Kx[pos] * p - S.Htdu[pos - w] * S.Kx[pos - w] * q);
    if (Hm[pos + 2 * w] > H_TINH && Hm[pos - 2 * w] > H_TINH) {
      q = (FS[pos + w] - FS[pos - w]) / (dX * 2);
      q = (S.tu[pos] + S.tu[pos - w]) * 0.5 * q * gamav;
    } else {
      q = 0;
    }
  }
  D = FS[pos] / (dT * 0.5) - q + p + (Sx / Hm[pos]);
}

}  // namespace hyd
