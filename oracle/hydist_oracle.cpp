// hydist_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A sequential FP64 CPU restatement of the Hydist_C time step (hydraulic ADI
// half-steps, wet/dry bookkeeping, smoothing, suspended-sediment sweeps) with
// the plain Thomas algorithm. It is the checker for the CUDA implementation:
// only tests/, the smoke check and bench.py's CPU-baseline leg load it. The
// product path never calls it.
//
// Every routine restates one reference kernel or device function and cites
// it as file:line (paths relative to the Hydist_C source tree). Each CUDA
// kernel's effect is reproduced as one sequential pass over the index range
// its launch shape reaches (engine.cpp launch sites). Where the reference's
// launch geometry silently skips cells only on meshes larger than 511 in a
// direction (engine.cpp:86-87, 184-185) the full range is used instead.
// Reference behaviour that is visible at every size is kept, including:
//   * the last end of a segment whose first end is open takes the first
//     end's discharge flag (UVZSolver_multithread.cpp:437-438);
//   * boundary series use segment 0 only (support_funcs.cpp:614-618);
//   * the second-half speed update skips row N (engine.cpp:259);
//   * the i-sweep of the concentration uses gamma_v = 0.98
//     (sediment_transport.cpp:247) and '&&' at the last end (:304);
//   * update_uvz never copies row N+1 / column M+1 (support_funcs.cpp:750).
// The extraction at an open last end reads the neighbour's velocity; in the
// reference that value is written by another thread of the same launch
// (UVZSolver_multithread.cpp:534, 598). race_new = 1 reads the freshly
// solved value, 0 the value from before the launch.
//
// Compile with -ffp-contract=off so that no multiply-add is fused.

#include "hydist_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int SEG = HYDIST_SEGMENT_LIMIT;
constexpr double kPI = 3.14159265358979323846;  // engine.h:13
constexpr double kEps = 1e-16;                  // UVZSolver_multithread.cpp:13

thread_local std::string g_err;

// Constant_Coeffs (engine.h:39-52), derived as Load_coeffs (loader.cpp:4-87).
struct Coeffs {
  double dX, dY, dT, dXbp, dYbp, dX2, dY2, dTchia2dX, dTchia2dY, HaiChiadT;
  double NANGDAY, H_TINH, heso, mu_mn, kenhhepng, kenhhepd;
  double NDnen, Tod, Toe, hstoe, ghtoe, Mbochat;
  double ro, ros, dm, muy, d90, Dorong, Sx;
  double CORIOLIS_FORCE, g, Ks, Windx, Windy, Ufr, Dxr, wss;
};

void derive(const HydistParams& p, Coeffs& c) {
  c.dX = p.dX;
  c.dY = p.dY;
  c.dT = p.dT;
  c.dXbp = c.dX * c.dX;
  c.dX2 = 2 * c.dX;
  c.dYbp = c.dY * c.dY;
  c.dY2 = 2 * c.dY;
  c.dTchia2dX = c.dT / c.dX2;
  c.dTchia2dY = c.dT / c.dY2;
  c.HaiChiadT = 2.0 / c.dT;
  c.kenhhepng = 0;
  c.kenhhepd = 0;
  c.NANGDAY = p.NANGDAY;
  c.H_TINH = p.H_TINH;
  c.heso = p.heso;
  c.mu_mn = p.mu_mn;
  c.NDnen = p.NDnen;
  c.Tod = p.Tod;
  c.Toe = p.Toe;
  c.hstoe = p.hstoe;
  c.ghtoe = p.ghtoe;
  c.Mbochat = p.Mbochat;
  c.ro = p.ro;
  c.ros = p.ros;
  c.dm = p.dm;
  c.d90 = p.d90;
  c.muy = p.muy;
  c.Dorong = p.Dorong;
  c.Sx = p.Sx;
  c.CORIOLIS_FORCE = p.CORIOLIS_FORCE;
  c.g = p.g;
  c.Ks = p.Ks >= 0 ? p.Ks : 2.5 * c.dm;  // loader.cpp:79
  // loader.cpp:81-82
  c.Windx = 0.0013 * (0.00075 + 0.000067 * std::fabs(p.Wind)) * std::fabs(p.Wind) * p.Wind *
            std::cos(p.huonggio * (kPI / 180));
  c.Windy = 0.0013 * (0.00075 + 0.000067 * std::fabs(p.Wind)) * std::fabs(p.Wind) * p.Wind *
            std::sin(p.huonggio * (kPI / 180));
  // loader.cpp:84-86 (operator order kept: g*(Sx-1)/muy*muy)
  c.Ufr = 0.25 * std::pow((c.Sx - 1) * c.g, 8.0 / 15.0) * std::pow(c.dm, 9.0 / 15.0) *
          std::pow(c.muy, -1.0 / 15.0);
  c.Dxr = c.dm * std::pow(c.g * (c.Sx - 1) / c.muy * c.muy, (1.0 / 3.0));
  c.wss = p.wss >= 0 ? p.wss
                     : 10 * c.muy / c.dm *
                           (std::sqrt(1 + 0.01 * (c.Sx - 1) * 9.81 * std::pow(c.dm, 3) /
                                              std::pow(c.muy, 2)) -
                            1);
}

struct Sim {
  int M = 0, N = 0, W = 0, H = 0, T = 0;
  Coeffs c{};
  HydistOptions o{};
  int race_new = 1;
  int nthreads = 1;
  double t = 0;

  std::vector<double> h, hsnham, visco, Fw;
  std::vector<double> bc[4], CC[4];  // up, down, left, right
  std::vector<int> btype;            // 4 x SEG, side-major
  int bienQ[4] = {0, 0, 0, 0};

  std::vector<double> u, v, z, tu, tv, tz, Hmoi, htaiz, htaiz_bd, Htdu, Htdv, Kx1, Ky1, Tsxw,
      Tsyw, FS, tFS, VTH, Kx, Ky, dH, Qbx, Qby;
  std::vector<int> khouot;
  std::vector<double> ubt, ubp, vbt, vbd, hi;
  double hmax_u = 0, hmax_d = 0, hmax_l = 0, hmax_r = 0;
  std::vector<int> daui, cuoii, moci, dauj, cuoij, mocj;
  bool seg_overflow = false;

  int id(int i, int j) const { return i * W + j; }

  std::vector<double>* field(int f) {
    switch (f) {
      case HYDIST_FIELD_U: return &u;
      case HYDIST_FIELD_V: return &v;
      case HYDIST_FIELD_Z: return &z;
      case HYDIST_FIELD_FS: return &FS;
      case HYDIST_FIELD_TFS: return &tFS;
      case HYDIST_FIELD_H_MOI: return &Hmoi;
      case HYDIST_FIELD_DH: return &dH;
      case HYDIST_FIELD_HTDU: return &Htdu;
      case HYDIST_FIELD_HTDV: return &Htdv;
      case HYDIST_FIELD_TU: return &tu;
      case HYDIST_FIELD_TV: return &tv;
      case HYDIST_FIELD_TZ: return &tz;
      case HYDIST_FIELD_KX1: return &Kx1;
      case HYDIST_FIELD_KY1: return &Ky1;
      case HYDIST_FIELD_VTH: return &VTH;
      case HYDIST_FIELD_KX: return &Kx;
      case HYDIST_FIELD_KY: return &Ky;
      case HYDIST_FIELD_H: return &h;
      case HYDIST_FIELD_HTAIZ: return &htaiz;
      case HYDIST_FIELD_QBX: return &Qbx;
      case HYDIST_FIELD_QBY: return &Qby;
      default: return nullptr;
    }
  }

  // ---------------------------------------------------------------- init
  // Onetime_init, support_funcs.cpp:21-69, over the launch of main.cpp:258-262.
  void onetime_init() {
    for (int i = 0; i < H; ++i) khouot[id(i, 0)] = 2;
    for (int j = 0; j < W; ++j) khouot[id(0, j)] = 2;
    for (int i = 1; i < H; ++i)
      for (int j = 1; j < W; ++j) khouot[id(i, j)] = 2;
    for (int i = 1; i <= N + 1; ++i)
      for (int j = 1; j <= M + 1; ++j) {
        if ((h[id(i - 1, j - 1)] + h[id(i - 1, j)] + h[id(i, j - 1)] + h[id(i, j)]) * 0.25 >
            c.NANGDAY) {
          khouot[id(i, j)] = 0;
          Hmoi[id(i, j)] = 0;
        }
      }
    for (int i = 1; i <= N; ++i)
      for (int j = 1; j <= M; ++j) {
        const int p = id(i, j);
        htaiz[p] = (h[id(i - 1, j - 1)] + h[id(i - 1, j)] + h[id(i, j - 1)] + h[p]) * 0.25;
        htaiz_bd[p] = htaiz[p];
        if (h[id(i, j - 1)] + h[p] != 0)
          Kx1[p] = c.g * std::pow((h[id(i, j - 1)] + h[p]) * 0.5, -2 * c.mu_mn) *
                   std::pow((hsnham[id(i, j - 1)] + hsnham[p]) * 0.5, 2);
        if (h[id(i - 1, j)] + h[p] != 0)
          Ky1[p] = c.g * std::pow((h[id(i - 1, j)] + h[p]) * 0.5, -2 * c.mu_mn) *
                   std::pow((hsnham[id(i - 1, j)] + hsnham[p]) * 0.5, 2);
      }
  }

  // The bed feedback (HydistOptions::bed_feedback; the reference computes
  // dH but never applies it): dH > 0 deepens the bed (the Exner balance of
  // sediment_transport.cpp:535, dH = dT/(1-porosity) (source + divergence)),
  // so htaiz = htaiz0 + dH at z points, a wet node's depth is its initial
  // depth plus the mean dH of the four cells around it (a node at NANGDAY
  // or below stays as it is), and Kx1, Ky1 follow from the new depths as in
  // Onetime_init (support_funcs.cpp:63-67). Once per step, after BedLoad.
  std::vector<double> h0, htaiz0;
  void keep_initial_bed() {
    h0 = h;
    htaiz0 = htaiz;
  }
  void bed_feedback() {
    for (int i = 0; i <= N + 1; ++i)
      for (int j = 0; j <= M + 1; ++j) {
        const int p = id(i, j);
        if (h0[p] > c.NANGDAY)
          h[p] = h0[p] + 0.25 * (dH[p] + dH[id(i + 1, j)] + dH[id(i, j + 1)] + dH[id(i + 1, j + 1)]);
      }
    for (int i = 1; i <= N; ++i)
      for (int j = 1; j <= M; ++j) {
        const int p = id(i, j);
        htaiz[p] = htaiz0[p] + dH[p];
        if (h[id(i, j - 1)] + h[p] != 0)
          Kx1[p] = c.g * std::pow((h[id(i, j - 1)] + h[p]) * 0.5, -2 * c.mu_mn) *
                   std::pow((hsnham[id(i, j - 1)] + hsnham[p]) * 0.5, 2);
        if (h[id(i - 1, j)] + h[p] != 0)
          Ky1[p] = c.g * std::pow((h[id(i - 1, j)] + h[p]) * 0.5, -2 * c.mu_mn) *
                   std::pow((hsnham[id(i - 1, j)] + hsnham[p]) * 0.5, 2);
      }
  }

  // preprocess_data, support_funcs.cpp:482-601 (one thread).
  void preprocess_data() {
    double* hu = hi.data();
    const double dX = c.dX, ND = c.NANGDAY, ros = c.ros;
    for (int k = 0; k < mocj[M]; ++k) {  // up: column M
      double sum = 0;
      for (int i = dauj[M * SEG + k]; i <= cuoij[M * SEG + k]; ++i) {
        hu[i] = (h[id(i, M)] + h[id(i - 1, M)]) / 2.0 - ND;
        sum += std::pow(hu[i], 5.0 / 3.0);
      }
      for (int i = dauj[M * SEG + k]; i <= cuoij[M * SEG + k]; ++i)
        hu[i] = std::pow(hu[i], 2.0 / 3.0) / (sum * dX);
    }
    double* hd = hu + (N + 3);
    for (int k = 0; k < mocj[2]; ++k) {  // down: column 2 (node column 1)
      double sum = 0;
      for (int i = dauj[2 * SEG + k]; i <= cuoij[2 * SEG + k]; ++i) {
        hd[i] = (h[id(i, 1)] + h[id(i - 1, 1)]) / 2.0 - ND;
        sum += std::pow(hd[i], 5.0 / 3.0);
      }
      for (int i = dauj[2 * SEG + k]; i <= cuoij[2 * SEG + k]; ++i)
        hd[i] = std::pow(hd[i], 2.0 / 3.0) / (sum * dX);
    }
    double* hl = hd + (N + 3);
    for (int k = 0; k < moci[2]; ++k) {  // left: row 2 (node row 1)
      double sum = 0;
      for (int j = daui[2 * SEG + k]; j <= cuoii[2 * SEG + k]; ++j) {
        hl[j] = (h[id(1, j)] + h[id(1, j - 1)]) / 2.0 - ND;
        sum += std::pow(hl[j], 5.0 / 3.0);
      }
      for (int j = daui[2 * SEG + k]; j <= cuoii[2 * SEG + k]; ++j)
        hl[j] = std::pow(hl[j], 2.0 / 3.0) / (sum * dX);
    }
    double* hr = hl + (M + 3);
    for (int k = 0; k < moci[N]; ++k) {  // right: row N
      double sum = 0;
      for (int j = daui[N * SEG + k]; j <= cuoii[N * SEG + k]; ++j) {
        hr[j] = (h[id(N, j)] + h[id(N, j - 1)]) / 2.0 - ND;
        sum += std::pow(hr[j], 5.0 / 3.0);
      }
      for (int j = daui[N * SEG + k]; j <= cuoii[N * SEG + k]; ++j)
        hr[j] = std::pow(hr[j], 2.0 / 3.0) / (sum * dX);
    }
    hmax_u = htaiz_bd[id(2, M)];
    hmax_d = htaiz_bd[id(2, 2)];
    for (int i = 3; i < N; ++i) {
      if (htaiz_bd[id(i, M)] > hmax_u) hmax_u = htaiz_bd[id(i, M)];
      if (htaiz_bd[id(i, 2)] > hmax_d) hmax_d = htaiz_bd[id(i, 2)];
    }
    hmax_l = htaiz_bd[id(2, 2)];
    hmax_r = htaiz_bd[id(N, 2)];
    for (int j = 3; j < M; ++j) {
      if (htaiz_bd[id(2, j)] > hmax_l) hmax_l = htaiz_bd[id(2, j)];
      if (htaiz_bd[id(N, j)] > hmax_r) hmax_r = htaiz_bd[id(N, j)];
    }
    if (hmax_u != 0) hmax_u = 1.0 / (ros * hmax_u);
    if (hmax_d != 0) hmax_d = 1.0 / (ros * hmax_d);
    if (hmax_l != 0) hmax_l = 1.0 / (ros * hmax_l);
    if (hmax_r != 0) hmax_r = 1.0 / (ros * hmax_r);
  }

  // ------------------------------------------------------ segment tables
  // Interpolate_FS_ng, support_funcs.cpp:191-213.
  void interpolate_fs_ng(int loc, int offset, int sign) {
    const double dT = c.dT, dX = c.dX;
    for (int j = 1; j < M; ++j) {
      if (tu[id(loc, j)] > 0) {
        const double deltaX = (u[id(loc, j)] + tu[id(loc, j)]) * 0.25 * dT;
        const double fi = offset + sign * (deltaX / dX);
        // a source row outside the mesh (only reachable once the state is
        // no longer finite) is skipped instead of read out of bounds
        if (!(fi > -1.0 && fi < (double)(H - 1))) continue;
        const int i = (int)fi;
        const int i_deltaX = (int)std::nearbyint(deltaX);
        const int i_dX = (int)std::nearbyint(dX);
        FS[id(loc, j)] = FS[id(i, j)] + sign * (FS[id(i + 1, j)] - FS[id(i, j)]) *
                                            (deltaX / dX - i_deltaX / i_dX);
      }
    }
  }
  // Interpolate_FS_d, support_funcs.cpp:215-237 (loops rows to M, :227).
  void interpolate_fs_d(int loc, int offset, int sign) {
    const double dT = c.dT, dY = c.dY;
    for (int i = 1; i < M && i < H; ++i) {
      if (tv[id(i, loc)] > 0) {
        const double deltaY = (v[id(i, loc)] + tv[id(i, loc)]) * 0.25 * dT;
        const double fj = offset + sign * (deltaY / dY);
        if (!(fj > -1.0 && fj < (double)(W - 1))) continue;
        const int j = (int)fj;
        const int j_deltaY = (int)std::nearbyint(deltaY);
        const int j_dY = (int)std::nearbyint(dY);
        FS[id(i, loc)] = FS[id(i, j + 1)] +
                         (FS[id(i, j + 1)] - FS[id(i, j)]) * (deltaY / dY - j_deltaY / j_dY);
      }
    }
  }

  // Scan of one line for wet runs: Find_Calculation_limits_Horizontal
  // (support_funcs.cpp:260-288) with stride 1, _Vertical (:313-341) with W.
  int scan_line(const int* k0, int stride, int lim, int* dau, int* cuoi) {
    int nseg = 0, start = 2, end = 0;
    auto K = [&](int q) { return k0[q * stride]; };
    while (start < lim) {
      if (K(start) != 0) {
        while (K(start) && start < lim) start++;
      }
      if (start + 1 == lim) start = lim;
      if (K(start) == 0 && start + 1 < lim) {
        if (nseg >= SEG) {
          seg_overflow = true;
          return nseg;
        }
        dau[nseg] = start;
        end = start;
        while (K(end) == 0 && end < lim) end++;
        if (K(end) != 0 && end <= lim) {
          cuoi[nseg] = end - 1;
          start = end;
          nseg++;
        } else {
          cuoi[nseg] = lim;
          start = lim;
          nseg++;
        }
      }
    }
    return nseg;
  }

  // the segment tables alone, from the mask as it stands (used after a
  // state is loaded from elsewhere)
  void rescan_segments() {
    for (int i = 2; i <= N; ++i)
      moci[i] = scan_line(&khouot[id(i, 0)], 1, M, &daui[i * SEG], &cuoii[i * SEG]);
    for (int j = 2; j <= M; ++j)
      mocj[j] = scan_line(&khouot[j], W, N, &dauj[j * SEG], &cuoij[j * SEG]);
  }

  void find_limits() {
    // Find_Calculation_limits_Horizontal, support_funcs.cpp:238-290
    interpolate_fs_ng(N, N - 1, -1);
    interpolate_fs_ng(2, 2, 1);
    for (int i = 2; i <= N; ++i)
      moci[i] = scan_line(&khouot[id(i, 0)], 1, M, &daui[i * SEG], &cuoii[i * SEG]);
    // Find_Calculation_limits_Vertical, support_funcs.cpp:293-343
    interpolate_fs_d(M, M - 1, -1);
    for (int j = 2; j <= M; ++j)
      mocj[j] = scan_line(&khouot[j], W, N, &dauj[j * SEG], &cuoij[j * SEG]);
  }

  // Htuongdoi, support_funcs.cpp:346-362.
  void htuongdoi() {
    for (int i = 1; i <= N; ++i)
      for (int j = 1; j <= M; ++j) {
        Htdu[id(i, j)] = (h[id(i, j - 1)] + h[id(i, j)] + z[id(i + 1, j)] + z[id(i, j)]) * 0.5;
        Htdv[id(i, j)] = (h[id(i - 1, j)] + h[id(i, j)] + z[id(i, j + 1)] + z[id(i, j)]) * 0.5;
      }
  }

  // ------------------------------------------------------------ boundary
  // Update_Boundary_Value / Boundary_value / FS_boundary,
  // support_funcs.cpp:603-728, launched by update_boundary_at_t
  // (engine.cpp:22-36) whose time argument is a float.
  void boundary(double t_in) {
    const double t = (double)(float)t_in;
    const int t1 = (int)(t / 3600);
    const double t2h = (t - (double)(3600.0f * (float)t1)) / 3600.0f;
    const double t2f = (t - (3600.0 * t1)) / 3600.0;
    const int mx = std::max(M, N);
    const double* hi_up = hi.data();
    const double* hi_down = hi_up + (N + 3);
    const double* hi_left = hi_down + (N + 3);
    const double* hi_right = hi_left + (M + 3);
    for (int i = 2; i <= mx; ++i) {
      // side: up (column M), down (column 2), left (row 2), right (row N)
      struct Side {
        bool isU;
        int loc, ext;
        const int *moc, *dau, *cuoi;
        const double* hiv;
        double* barr;
        double hmax;
      } sides[4] = {
          {false, M, M + 1, mocj.data(), dauj.data(), cuoij.data(), hi_up, vbt.data(), hmax_u},
          {false, 2, 1, mocj.data(), dauj.data(), cuoij.data(), hi_down, vbd.data(), hmax_d},
          {true, 2, 1, moci.data(), daui.data(), cuoii.data(), hi_left, ubt.data(), hmax_l},
          {true, N, N + 1, moci.data(), daui.data(), cuoii.data(), hi_right, ubp.data(), hmax_r}};
      for (int s = 0; s < 4; ++s) {
        const Side& S = sides[s];
        const int* bt = &btype[s * SEG];
        // Boundary_value: only segment 0 is tested (support_funcs.cpp:614-618)
        int seg = -1;
        if (S.moc[S.loc] > 0) {
          if (S.dau[S.loc * SEG] <= i && i <= S.cuoi[S.loc * SEG]) seg = 0;
        }
        if (seg == -1) continue;
        const double* B = bc[s].data();
        const double val = B[seg * T + t1] * (1.0f - t2h) + B[seg * T + t1 + 1] * t2h;
        if (bt[seg] == 2) {
          S.barr[i] = val * S.hiv[i];
        } else {
          if (S.isU) {
            tz[id(S.loc, i)] = val;
            tz[id(S.ext, i)] = val;
          } else {
            tz[id(i, S.loc)] = val;
            tz[id(i, S.ext)] = val;
          }
        }
        // FS_boundary (support_funcs.cpp:642-677)
        if (bt[seg] != 2) continue;
        const double* C = CC[s].data();
        const double cv = C[seg * T + t1] * (1.0 - t2f) + C[seg * T + t1 + 1] * t2f;
        const int ii = S.isU ? S.loc : i;
        const int jj = S.isU ? i : S.loc;
        FS[id(ii, jj)] = cv * htaiz_bd[id(ii, jj)] * S.hmax;
      }
    }
  }

  // The narrow-channel standing wave: boundary_up / boundary_down /
  // boundary_left / boundary_right (support_funcs.cpp:366-478), whose calls
  // the reference keeps commented out in update_boundary_at_t
  // (engine.cpp:25-28). Each walks the first wet segment of its side's line
  // (boundary_right from row 2's first start to row N's first end, as
  // written); a side without a wet segment is skipped.
  void channel_wave(double t_in) {
    const double t = (double)(float)t_in;
    const double PI_ = 3.14159265358979323846;
    const double ct = std::cos(2 * PI_ / 27.75 * t);
    if (mocj[M] > 0)  // up: column M, bienQ[0] not consulted
      for (int i = dauj[M * SEG]; i <= cuoij[M * SEG]; ++i) {
        tz[id(i, M)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * (100 - c.dY / 2));
        tz[id(i, M + 1)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * (100 + c.dY / 2));
      }
    if (mocj[2] > 0)  // down: column 2
      for (int i = dauj[2 * SEG]; i <= cuoij[2 * SEG]; ++i) {
        if (bienQ[1]) {
          vbd[i] = 0;
        } else {
          tz[id(i, 2)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * c.dY / 2);
          tz[id(i, 1)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * (-c.dY) / 2);
        }
      }
    if (moci[2] > 0)  // left: row 2
      for (int j = daui[2 * SEG]; j <= cuoii[2 * SEG]; ++j) {
        if (bienQ[2]) {
          ubt[j] = 0;
        } else {
          tz[id(2, j)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * c.dX / 2);
          tz[id(1, j)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * (-c.dX) / 2);
        }
      }
    if (moci[2] > 0 && moci[N] > 0)  // right: row N
      for (int j = daui[2 * SEG]; j <= cuoii[N * SEG]; ++j) {
        if (bienQ[3]) {
          ubp[j] = 0;
        } else {
          tz[id(N, j)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * (100 - c.dX / 2));
          tz[id(N + 1, j)] = 0.01 * ct * std::cos(2 * (PI_ / 100) * (100 + c.dX / 2));
        }
      }
  }

  // update_boundary_at_t (engine.cpp:22-36): the series outside channel
  // mode; in channel mode nothing, or the standing wave when asked for
  bool channel() const { return (o.kenhhepd != 0) != (o.kenhhepng != 0); }
  void update_boundary(double t_in) {
    if (!channel()) boundary(t_in);
    else if (o.channel_wave) channel_wave(t_in);
  }

  // -------------------------------------------------- segment end flags
  // locate_segment_v (support_funcs.cpp:810-830) for row i.
  void ends_v(int i, int first, int last, bool& b1, bool& b2) const {
    b1 = (first > 2) || ((first == 2) && ((h[id(i, first - 1)] + h[id(i - 1, first - 1)]) * 0.5 ==
                                          c.NANGDAY));
    b2 = (last < M) ||
         ((last == M) && ((h[id(i, last)] + h[id(i - 1, last)]) * 0.5 == c.NANGDAY));
  }
  // locate_segment_u (support_funcs.cpp:832-858) for column j.
  void ends_u(int j, int first, int last, bool& b1, bool& b2) const {
    b1 = (first > 2) ||
         ((first == 2) && ((h[id(1, j)] + h[id(1, j - 1)]) * 0.5 == c.NANGDAY));
    b2 = (last < N) || ((last == N) && ((h[id(N, j)] + h[id(N, j - 1)]) * 0.5 == c.NANGDAY));
  }

  // ------------------------------------------------------ Thomas solver
  // tridiag, UVZSolver_multithread.cpp:19-43 (no pivoting).
  static void thomas(int sn, const double* AA, const double* BB, const double* CC,
                     const double* DD, double* x, std::vector<double>& Ap,
                     std::vector<double>& Bp) {
    if (sn < 0) return;
    if (sn == 0) {
      x[0] = DD[0] / BB[0];
      return;
    }
    if ((int)Ap.size() < sn + 1) {
      Ap.resize(sn + 1);
      Bp.resize(sn + 1);
    }
    Ap[0] = -CC[0] / BB[0];
    Bp[0] = DD[0] / BB[0];
    for (int i = 1; i < sn; ++i) {
      const double ep = AA[i] * Ap[i - 1] + BB[i];
      Ap[i] = -CC[i] / ep;
      Bp[i] = (DD[i] - (AA[i] * Bp[i - 1])) / ep;
    }
    x[sn] = (DD[sn] - (AA[sn] * Bp[sn - 1])) / (BB[sn] + (AA[sn] * Ap[sn - 1]));
    for (int i = sn - 1; i >= 0; --i) x[i] = Bp[i] + (Ap[i] * x[i + 1]);
  }

  // Per-line work buffers for one hydraulic sweep.
  struct LineBuf {
    std::vector<double> f1, f2, f3, f5, a1, b1, c1, d1, a2, c2, d2, AA, BB, CC, DD, x, Ap, Bp;
    std::vector<double> old_vel;
    void size(int n_cells, int n_unk) {
      for (auto* vp : {&f1, &f2, &f3, &f5, &a1, &b1, &c1, &d1, &a2, &c2, &d2, &old_vel})
        vp->assign(n_cells, 0.0);
      for (auto* vp : {&AA, &BB, &CC, &DD, &x}) vp->assign(n_unk, 0.0);
    }
  };

  // _calculate_abcd, UVZSolver_multithread.cpp:280-342, for one segment.
  static void calc_abcd(LineBuf& L, int first, int last, double f4, bool br1, bool br2) {
    double *a1 = L.a1.data(), *b1 = L.b1.data(), *c1 = L.c1.data(), *d1 = L.d1.data();
    const double *a2 = L.a2.data(), *c2 = L.c2.data(), *d2 = L.d2.data(), *f1 = L.f1.data(),
                 *f2 = L.f2.data(), *f3 = L.f3.data(), *f5 = L.f5.data();
    if (last - 1 > first) {
      // row `last` would read coefficients past the segment; it never enters
      // the system, so only [first, last-1] is formed.
      for (int j = first; j <= last - 1; ++j) {
        a1[j] = f4 - f1[j] / a2[j];
        c1[j] = -f4 - (f3[j] / c2[j + 1]);
        b1[j] = f2[j] - (f1[j] * c2[j] / a2[j]) - (f3[j] * a2[j + 1] / c2[j + 1]);
        d1[j] = f5[j] - (f1[j] * d2[j] / a2[j]) - (f3[j] * d2[j + 1] / c2[j + 1]);
      }
      if (br1) {
        a1[first] = f4;
        b1[first] = f2[first] - (f3[first] * a2[first + 1] / c2[first + 1]);
        c1[first] = -f4 - (f3[first] / c2[first + 1]);
        d1[first] = f5[first] - (f3[first] * d2[first + 1] / c2[first + 1]);
      }
      if (br2) {
        a1[last - 1] = f4 - f1[last - 1] / a2[last - 1];
        b1[last - 1] = f2[last - 1] - (f1[last - 1] * c2[last - 1] / a2[last - 1]);
        c1[last - 1] = -f4;
        d1[last - 1] = f5[last - 1] - (f1[last - 1] * d2[last - 1] / a2[last - 1]);
      }
    } else {
      a1[first] = f4;
      b1[first] = f2[first];
      d1[first] = f5[first];
      c1[first] = -f4;
    }
  }

  // _calculate_matrix_coeff + bienrandau/bienlongdau,
  // UVZSolver_multithread.cpp:110-139, 345-470. Returns sn.
  static int calc_matrix(LineBuf& L, int first, int last, bool br1, bool br2, double ubt_vbd,
                         double ubp_vbt, double TZ_r, double TZ_l, bool q1, bool q2, int dkfr) {
    double *AA = L.AA.data(), *BB = L.BB.data(), *CC = L.CC.data(), *DD = L.DD.data();
    const double *a1 = L.a1.data(), *b1 = L.b1.data(), *c1 = L.c1.data(), *d1 = L.d1.data(),
                 *a2 = L.a2.data(), *c2 = L.c2.data(), *d2 = L.d2.data();
    const int off = first * 2;
    int sn = 2 * (last - first);
    auto ran = [&](int j) {  // bienrandau
      AA[j * 2] = a2[j];
      AA[j * 2 + 1] = a1[j];
      BB[j * 2] = 1;
      BB[j * 2 + 1] = b1[j];
      CC[j * 2] = c2[j];
      CC[j * 2 + 1] = c1[j];
      DD[j * 2] = d2[j];
      DD[j * 2 + 1] = d1[j];
    };
    auto lon = [&](int j) {  // bienlongdau
      AA[j * 2] = a1[j];
      AA[j * 2 + 1] = a2[j + 1];
      BB[j * 2] = b1[j];
      BB[j * 2 + 1] = 1;
      CC[j * 2] = c1[j];
      CC[j * 2 + 1] = c2[j + 1];
      DD[j * 2] = d1[j];
      DD[j * 2 + 1] = d2[j + 1];
    };
    // rows 2*last+1 (bienrandau) and 2*last, 2*last+1 (bienlongdau) use
    // coefficients past the segment and never enter the system: not formed.
    if (br1) {
      for (int j = first; j <= last; ++j) {
        if (j < last) {
          ran(j);
        } else {
          AA[j * 2] = a2[j];
          BB[j * 2] = 1;
          CC[j * 2] = c2[j];
          DD[j * 2] = d2[j];
        }
      }
      DD[off] = d2[first];
      if (!br2) {
        if (q2 && last == dkfr) {
          AA[sn + off] = a2[last];
          BB[sn + off] = 1;
          DD[sn + off] = d2[last] - c2[last] * ubp_vbt;
        } else {
          sn--;
          AA[sn + off] = a1[last - 1];
          BB[sn + off] = b1[last - 1];
          DD[sn + off] = d1[last - 1] - c1[last - 1] * TZ_r;
        }
      } else {
        AA[sn + off] = a2[last];
        BB[sn + off] = 1;
        DD[sn + off] = d2[last];
      }
    } else {
      bool isBienran;
      if (q1 && first == 2) {
        for (int j = first; j <= last; ++j) {
          if (j < last) {
            ran(j);
          } else {
            AA[j * 2] = a2[j];
            BB[j * 2] = 1;
            CC[j * 2] = c2[j];
            DD[j * 2] = d2[j];
          }
        }
        DD[off] = d2[first] - a2[first] * ubt_vbd;
        isBienran = true;
      } else {
        for (int j = first; j < last; ++j) lon(j);
        BB[off] = b1[first];
        CC[off] = c1[first];
        DD[off] = d1[first] - a1[first] * TZ_l;
        isBienran = false;
      }
      if (!br2) {
        if (q1 && last == dkfr) {  // first end's flag (UVZSolver_multithread.cpp:438)
          if (!isBienran) sn--;
          AA[sn + off] = a2[last];
          BB[sn + off] = 1;
          DD[sn + off] = d2[last] - c2[last] * ubp_vbt;
        } else {
          sn--;
          if (!isBienran) sn -= 1;
          AA[sn + off] = a1[last - 1];
          BB[sn + off] = b1[last - 1];
          DD[sn + off] = d1[last - 1] - c1[last - 1] * TZ_r;
        }
      } else {
        if (!isBienran) sn--;
        AA[sn + off] = a2[last];
        BB[sn + off] = 1;
        DD[sn + off] = d2[last];
      }
    }
    return sn;
  }

  // ---------------------------------------------- UZ half-step (x sweep)
  // _uzSolver_calculate_preindex, UVZSolver_multithread.cpp:210-278.
  void uz_preindex(LineBuf& L, int i, int j) const {
    const double H_TINH = c.H_TINH, dT = c.dT, dXbp = c.dXbp, dYbp = c.dYbp, dY2 = c.dY2,
                 dTchia2dY = c.dTchia2dY, dTchia2dX = c.dTchia2dX, Windx = c.Windx,
                 COR = c.CORIOLIS_FORCE;
    const int w = W;
    double p = 0.0, q = 0.0;
    const double vtb = (v[i * w + j - 1] + v[i * w + j] + v[(i + 1) * w + j - 1] +
                        v[(i + 1) * w + j]) *
                       0.25;
    const double uu = u[i * w + j], VI = visco[i * w + j];
    L.f1[i] = dTchia2dX * uu + VI * dT / dXbp;
    L.f2[i] = -(2 + Kx1[i * w + j] * dT * std::sqrt(uu * uu + vtb * vtb) / Htdu[i * w + j] +
                (2 * dT * VI) / dXbp);
    L.f3[i] = dT * VI / dXbp - dTchia2dX * uu;
    if (Hmoi[i * w + j - 1] <= H_TINH) {
      if (vtb < 0) {
        p = vtb * (-3 * uu + 4 * u[i * w + j + 1] - u[i * w + j + 2]) / dY2;
        q = (uu - 2 * u[i * w + j + 1] + u[i * w + j + 2]) / dYbp;
      }
    } else {
      if (Hmoi[i * w + j + 1] <= H_TINH) {
        if ((Hmoi[i * w + j - 2] > H_TINH) && (vtb > 0)) {
          p = vtb * (3 * uu - 4 * u[i * w + j - 1] + u[i * w + j - 2]) / dY2;
          q = (uu - 2 * u[i * w + j - 1] + u[i * w + j - 2]) / dYbp;
        }
      } else {
        p = vtb * (u[i * w + j + 1] - u[i * w + j - 1]) / dY2;
        q = (u[i * w + j + 1] - 2 * uu + u[i * w + j - 1]) / dYbp;
      }
    }
    L.f5[i] = -2 * uu + dT * p - dT * COR * vtb - dT * VI * q -
              dT * (Windx - Tsxw[i * w + j]) / Htdu[i * w + j];
    L.c2[i] = dTchia2dX * Htdu[i * w + j];
    L.a2[i] = -dTchia2dX * Htdu[(i - 1) * w + j];
    L.d2[i] = z[i * w + j] -
              dTchia2dY * (Htdv[i * w + j] * v[i * w + j] - Htdv[i * w + j - 1] * v[i * w + j - 1]);
  }

  // UZ sweep of column j: preindex, abcd, matrix, tridiagSolver, extract
  // (engine.cpp:91-104).
  void uz_column(LineBuf& L, int j) {
    const int w = W;
    const double f4 = 2 * c.g * c.dTchia2dX;
    for (int k = 0; k < mocj[j]; ++k) {
      const int first = dauj[j * SEG + k], last = cuoij[j * SEG + k];
      bool br1, br2;
      ends_u(j, first, last, br1, br2);
      for (int i = first; i <= last; ++i) uz_preindex(L, i, j);
      calc_abcd(L, first, last, f4, br1, br2);
      const int sn = calc_matrix(L, first, last, br1, br2, ubt[j], ubp[j], tz[last * w + j],
                                 tz[first * w + j], bienQ[2], bienQ[3], N);
      const int pos = 2 * first;
      thomas(sn, &L.AA[pos], &L.BB[pos], &L.CC[pos], &L.DD[pos], &L.x[pos], L.Ap, L.Bp);
      // a degenerate one-cell system (sn < 0) is not solved; its ends read 0
      if (sn < 0 && pos + sn >= 0) L.x[pos + sn] = 0.0;
      // _uzSolver_extract_solution, UVZSolver_multithread.cpp:547-603
      const double* x = L.x.data();
      const double tu_prev = (last - 1 >= 0) ? tu[(last - 1) * w + j] : 0.0;
      for (int i = first; i <= last; ++i) {
        if (i < last) {
          if (br1) {
            tz[i * w + j] = x[2 * i];
            tu[i * w + j] = x[2 * i + 1];
            tu[(first - 1) * w + j] = 0;
          } else if (bienQ[2] && first == 2) {
            tz[i * w + j] = x[2 * i];
            tu[i * w + j] = x[2 * i + 1];
            tu[(first - 1) * w + j] = ubt[j];
          } else {
            if (i == first) {
              tu[first * w + j] = x[first * 2];
              tu[(first - 1) * w + j] =
                  (L.d2[first] - tz[first * w + j] - L.c2[first] * tu[first * w + j]) /
                  L.a2[first];
            } else {
              tz[i * w + j] = x[2 * i - 1];
              tu[i * w + j] = x[2 * i];
            }
          }
        } else {
          if (br2) {
            tu[last * w + j] = 0;
            tz[last * w + j] = x[first * 2 + sn];
          } else if (bienQ[3] && last == N) {
            tu[last * w + j] = ubp[j];
            tz[last * w + j] = x[first * 2 + sn];
          } else {
            const double nb = race_new ? tu[(last - 1) * w + j] : tu_prev;
            tu[last * w + j] = (L.d2[last] - L.a2[last] * nb - tz[last * w + j]) / L.c2[last];
          }
        }
      }
    }
  }

  // ---------------------------------------------- VZ half-step (y sweep)
  // _vzSolver_calculate_preindex, UVZSolver_multithread.cpp:142-208.
  void vz_preindex(LineBuf& L, int i, int j) const {
    const double H_TINH = c.H_TINH, dT = c.dT, dXbp = c.dXbp, dYbp = c.dYbp, dX2 = c.dX2,
                 dTchia2dY = c.dTchia2dY, dTchia2dX = c.dTchia2dX, Windy = c.Windy,
                 COR = c.CORIOLIS_FORCE;
    const int w = W;
    double p = 0.0, q = 0.0;
    const double utb = (u[(i - 1) * w + j] + u[i * w + j] + u[(i - 1) * w + j + 1] +
                        u[i * w + j + 1]) *
                       0.25;
    const double vv = v[i * w + j], VI = visco[i * w + j];
    L.f1[j] = dTchia2dY * vv + VI * dT / dYbp;
    L.f2[j] = -(2 + Ky1[i * w + j] * dT * std::sqrt(vv * vv + utb * utb) / Htdv[i * w + j] +
                (2 * dT * VI) / dYbp);
    L.f3[j] = dT * VI / dYbp - dTchia2dY * vv;
    if (Hmoi[(i - 1) * w + j] <= H_TINH) {
      if (utb < 0) {
        q = utb * (-3 * vv + 4 * v[(i + 1) * w + j] - v[(i + 2) * w + j]) / dX2;
        p = (vv - 2 * v[(i + 1) * w + j] + v[(i + 2) * w + j]) / dXbp;
      }
    } else {
      if (Hmoi[(i + 1) * w + j] <= H_TINH) {
        if ((Hmoi[(i - 2) * w + j] > H_TINH) && (utb > 0)) {
          q = utb * (3 * vv - 4 * v[(i - 1) * w + j] + v[(i - 2) * w + j]) / dX2;
          p = (vv - 2 * v[(i - 1) * w + j] + v[(i - 2) * w + j]) / dXbp;
        }
      } else {
        q = utb * (v[(i + 1) * w + j] - v[(i - 1) * w + j]) / dX2;
        p = (v[(i + 1) * w + j] - 2 * vv + v[(i - 1) * w + j]) / dXbp;
      }
    }
    L.f5[j] = -2 * vv + dT * q + dT * COR * utb - dT * VI * p -
              dT * (Windy - Tsyw[i * w + j]) / Htdv[i * w + j];
    L.c2[j] = dTchia2dY * Htdv[i * w + j];
    L.a2[j] = -dTchia2dY * Htdv[i * w + j - 1];
    L.d2[j] = z[i * w + j] -
              dTchia2dX * (Htdu[i * w + j] * u[i * w + j] - Htdu[(i - 1) * w + j] * u[(i - 1) * w + j]);
  }

  // VZ sweep of row i (engine.cpp:196-208); extraction reaches columns
  // j <= N only (VZSolver_extract_solution, UVZSolver_multithread.cpp:851).
  void vz_row(LineBuf& L, int i) {
    const int w = W;
    const double f4 = 2 * c.g * c.dTchia2dY;
    for (int k = 0; k < moci[i]; ++k) {
      const int first = daui[i * SEG + k], last = cuoii[i * SEG + k];
      bool br1, br2;
      ends_v(i, first, last, br1, br2);
      for (int j = first; j <= last; ++j) vz_preindex(L, i, j);
      calc_abcd(L, first, last, f4, br1, br2);
      const int sn = calc_matrix(L, first, last, br1, br2, vbd[i], vbt[i], tz[i * w + last],
                                 tz[i * w + first], bienQ[1], bienQ[0], M);
      const int pos = 2 * first;
      thomas(sn, &L.AA[pos], &L.BB[pos], &L.CC[pos], &L.DD[pos], &L.x[pos], L.Ap, L.Bp);
      if (sn < 0 && pos + sn >= 0) L.x[pos + sn] = 0.0;
      // _vzSolver_extract_solution, UVZSolver_multithread.cpp:472-544
      const double* x = L.x.data();
      const double tv_prev = tv[i * w + last - 1];
      for (int j = first; j <= last; ++j) {
        if (j > N) break;
        if (j < last) {
          if (br1) {
            tz[i * w + j] = x[2 * j];
            tv[i * w + j] = x[2 * j + 1];
            tv[i * w + first - 1] = 0;
          } else if (bienQ[1] && first == 2) {
            tz[i * w + j] = x[2 * j];
            tv[i * w + j] = x[2 * j + 1];
            tv[i * w + first - 1] = vbd[i];
          } else {
            if (j == first) {
              tv[i * w + first] = x[2 * first];
              tv[i * w + first - 1] =
                  (L.d2[first] - tz[i * w + first] - L.c2[first] * tv[i * w + first]) /
                  L.a2[first];
            } else {
              tz[i * w + j] = x[2 * j - 1];
              tv[i * w + j] = x[2 * j];
            }
          }
        } else {
          if (br2) {
            tv[i * w + last] = 0;
            tz[i * w + last] = x[first * 2 + sn];
          } else if (bienQ[0] && last == M) {
            tv[i * w + last] = vbt[i];
            tz[i * w + last] = x[2 * first + sn];
          } else {
            const double nb = race_new ? tv[i * w + last - 1] : tv_prev;
            tv[i * w + last] = (L.d2[last] - L.a2[last] * nb - tz[i * w + last]) / L.c2[last];
          }
        }
      }
    }
  }

  // ------------------------------------------------------- smoothing
  // Normalize + _normalize + update_buffer, support_funcs.cpp:761-808.
  void normalize(bool isU, std::vector<double>& tmp) {
    std::vector<double>& val = isU ? tu : tv;
    const int close = isU ? W : 1, far = isU ? 1 : W;
    const double coeff = c.heso;
    tmp = val;
    for (int i = 2; i <= N; ++i)
      for (int j = 2; j <= M; ++j) {
        const int g = id(i, j);
        if (val[g] != 0) {
          int count = 2;
          double nb = val[g - close] + val[g + close];
          if (khouot[g - far] == 0) {
            nb += val[g - far];
            count++;
          }
          if (khouot[g + far] == 0) {
            nb += val[g + far];
            count++;
          }
          tmp[g] = tmp[g] * coeff + (1 - coeff) * nb / count;
        }
      }
    for (int i = 2; i <= N; ++i)
      for (int j = 2; j <= M; ++j) val[id(i, j)] = tmp[id(i, j)];
  }

  // ------------------------------------------------ explicit updates
  // vSolver, UVZSolver_multithread.cpp:607-663, driven by solveV (:961-978).
  void solve_v() {
    const double H_TINH = c.H_TINH, dY2 = c.dY2, dX2 = c.dX2, dY = c.dY, COR = c.CORIOLIS_FORCE,
                 Windy = c.Windy, dXbp = c.dXbp, dYbp = c.dYbp, g = c.g, HaiChiadT = c.HaiChiadT;
    const int off = W;
    for (int row = 2; row <= N; ++row)
      for (int k = 0; k < moci[row]; ++k) {
        const int first = daui[row * SEG + k], last = cuoii[row * SEG + k];
        if (first >= last) continue;
        for (int col = first; col < last; ++col) {
          double p, q = 0, tmp = 0;
          const double utb = (u[(row - 1) * off + col] + u[row * off + col] +
                              u[(row - 1) * off + col + 1] + u[row * off + col + 1]) *
                             0.25;
          const double t_utb = (tu[(row - 1) * off + col] + tu[row * off + col] +
                                tu[(row - 1) * off + col + 1] + tu[row * off + col + 1]) *
                               0.25;
          const double vv = v[row * off + col];
          p = (v[row * off + col + 1] - v[row * off + col - 1]) / dY2;
          p = HaiChiadT + p +
              Ky1[row * off + col] * std::sqrt(utb * utb + vv * vv) / Htdv[row * off + col];
          if (Hmoi[(row - 1) * off + col] <= H_TINH) {
            if (utb < 0) {
              q = t_utb * (-3 * vv + 4 * v[(row + 1) * off + col] - v[(row + 2) * off + col]) /
                  dX2;
              tmp = (vv - 2 * v[(row + 1) * off + col] + v[(row + 2) * off + col]) / dXbp;
            }
          } else {
            if (Hmoi[(row + 1) * off + col] <= H_TINH) {
              if ((Hmoi[(row - 2) * off + col] > H_TINH) && (utb > 0)) {
                q = t_utb * (3 * vv - 4 * v[(row - 1) * off + col] + v[(row - 2) * off + col]) /
                    dX2;
                tmp = (vv - 2 * v[(row - 1) * off + col] + v[(row - 2) * off + col]) / dXbp;
              }
            } else {
              q = t_utb * (v[(row + 1) * off + col] - v[(row - 1) * off + col]) / dX2;
              tmp = (v[(row + 1) * off + col] - 2 * vv + v[(row - 1) * off + col]) / dXbp;
            }
          }
          q = HaiChiadT * vv - q - COR * t_utb;
          q = (q - g * (z[row * off + col + 1] - z[row * off + col]) / dY +
               visco[row * off + col] *
                   (tmp + (v[row * off + col + 1] - 2 * vv + v[row * off + col - 1]) / dYbp)) +
              (Windy - Tsyw[row * off + col]) / Htdv[row * off + col];
          tv[row * off + col] = q / p;
        }
      }
  }

  // uSolver, UVZSolver_multithread.cpp:724-795, driven by solveU (:938-959).
  // uSolver reads dX and Windx from coeffs->dY and coeffs->Windy (:731,734).
  void solve_u() {
    const double H_TINH = c.H_TINH, dX = c.dY, dY = c.dY, COR = c.CORIOLIS_FORCE,
                 Windx = c.Windy, g = c.g, HaiChiadT = c.HaiChiadT;
    const int off = W;
    for (int col = 2; col <= M; ++col)
      for (int k = 0; k < mocj[col]; ++k) {
        const int first = dauj[col * SEG + k], last = cuoij[col * SEG + k];
        for (int row = std::max(first, 1); row < last && row <= N; ++row) {
          double p, q = 0, tmp = 0;
          const int ij = row * off + col, i1j = ij + off;
          const double vtb = (v[ij - 1] + v[ij] + v[i1j - 1] + v[i1j]) * 0.25;
          const double t_vtb = (tv[ij - 1] + tv[ij] + tv[i1j - 1] + tv[i1j]) * 0.25;
          p = (u[i1j] - u[(row - 1) * off + col]) / (dX * 2);
          p = (HaiChiadT + p + Kx1[ij] * std::sqrt(vtb * vtb + u[ij] * u[ij]) / Htdu[ij]);
          if (Hmoi[ij - 1] <= H_TINH) {
            if (vtb < 0) {
              q = t_vtb * (-3 * u[ij] + 4 * u[ij + 1] - u[ij + 2]) / (dY * 2);
              tmp = (u[ij] - 2 * u[ij + 1] + u[ij + 2]) / (dY * dY);
            }
          } else {
            if (Hmoi[ij + 1] <= H_TINH) {
              if ((Hmoi[ij - 2] > H_TINH) && (vtb > 0)) {
                q = t_vtb * (3 * u[ij] - 4 * u[ij - 1] + u[ij - 2]) / (dY * 2);
                tmp = (u[ij] - 2 * u[ij - 1] + u[ij - 2]) / (dY * dY);
              }
            } else {
              q = t_vtb * (u[ij + 1] - u[ij - 1]) / (dY * 2);
              tmp = (u[ij + 1] - 2 * u[ij] + u[ij - 1]) / (dY * dY);
            }
          }
          q = HaiChiadT * u[ij] - q + COR * t_vtb;
          q = (q - g * (z[i1j] - z[ij]) / dX +
               visco[ij] * (tmp + (u[i1j] - 2 * u[ij] + u[(row - 1) * off + col]) / (dX * dX))) +
              (Windx - Tsxw[ij]) / Htdu[ij];
          tu[ij] = q / p;
        }
      }
  }

  // update_margin_elem_V, UVZSolver_multithread.cpp:1018-1060.
  void margin_v() {
    const int w = W;
    for (int i = 2; i <= N; ++i)
      for (int k = 0; k < moci[i]; ++k) {
        const int first = daui[i * SEG + k], last = cuoii[i * SEG + k];
        const bool br1 =
            (first > 2) ||
            ((first == 2) &&
             (std::fabs((h[i * w + first - 1] + h[(i - 1) * w + first - 1]) * 0.5 - c.NANGDAY) <
              kEps));
        const bool br2 =
            (last < M) ||
            ((last == M) &&
             (std::fabs((h[i * w + last] + h[(i - 1) * w + last]) * 0.5 - c.NANGDAY) < kEps));
        if (br1)
          tv[i * w + first - 1] = 0;
        else
          tv[i * w + first - 1] = 2 * tv[i * w + first] - tv[i * w + first + 1];
        if (br2)
          tv[i * w + last] = 0;
        else
          tv[i * w + last] = 2 * tv[i * w + last - 1] - tv[i * w + last - 2];
      }
  }

  // update_margin_elem_U, UVZSolver_multithread.cpp:980-1016.
  void margin_u() {
    const int w = W;
    for (int j = 2; j <= M; ++j)
      for (int k = 0; k < mocj[j]; ++k) {
        const int first = dauj[j * SEG + k], last = cuoij[j * SEG + k];
        const bool br1 =
            (first > 2) ||
            ((first == 2) &&
             (std::fabs((h[1 * w + j] + h[1 * w + j - 1]) * 0.5 - c.NANGDAY) < kEps));
        const bool br2 =
            (last < N) ||
            ((last == N) && (std::fabs((h[N * w + j] + h[N * w + j - 1]) * 0.5 - c.NANGDAY) < kEps));
        if (br1)
          tu[(first - 1) * w + j] = 0;
        else
          tu[(first - 1) * w + j] = 2 * tu[first * w + j] - tu[(first + 1) * w + j];
        if (br2)
          tu[last * w + j] = 0;
        else
          tu[last * w + j] = 2 * tu[(last - 1) * w + j] - tu[(last - 2) * w + j];
      }
  }

  // update_h_moi, support_funcs.cpp:71-86.
  void update_h_moi() {
    for (int i = 1; i <= N; ++i)
      for (int j = 1; j <= M; ++j) {
        const int g = id(i, j);
        if (khouot[g] == 0) Hmoi[g] = htaiz[g] + tz[g];
      }
  }

  // update_uvz, support_funcs.cpp:732-759 (rows/columns 0..N / 0..M).
  void update_uvz() {
    for (int i = 0; i <= N; ++i)
      for (int j = 0; j <= M; ++j) {
        const int g = id(i, j);
        z[g] = tz[g];
        u[g] = tu[g] * (1 - c.kenhhepd);
        v[g] = tv[g] * (1 - c.kenhhepng);
      }
  }

  // Reset_states_vertical, support_funcs.cpp:142-188.
  void reset_states_vertical() {
    const int off = W;
    for (int j = 1; j <= M; ++j) {
      for (int i = 2; i <= N; ++i) {
        if (tz[i * off + j] > z[i * off + j]) {
          if (khouot[(i - 1) * off + j] == 1) {
            tz[(i - 1) * off + j] = tz[i * off + j];
            Hmoi[(i - 1) * off + j] = htaiz[(i - 1) * off + j] + tz[i * off + j];
            khouot[(i - 1) * off + j] = 0;
            FS[(i - 1) * off + j] = FS[i * off + j];
          }
          if (khouot[(i + 1) * off + j] == 1) {
            tz[(i + 1) * off + j] = tz[i * off + j];
            Hmoi[(i + 1) * off + j] = htaiz[(i + 1) * off + j] + tz[i * off + j];
            khouot[(i + 1) * off + j] = 0;
            FS[(i + 1) * off + j] = FS[i * off + j];
          }
        }
      }
      for (int i = 2; i <= N; ++i) {
        if ((khouot[i * off + j] == 0) && (Hmoi[i * off + j] <= c.H_TINH)) {
          tu[(i - 1) * off + j] = 0;
          tu[i * off + j] = 0;
          tv[i * off + j - 1] = 0;
          tv[i * off + j] = 0;
          khouot[i * off + j] = 1;
          FS[i * off + j] = 0;
        }
      }
    }
  }

  // Reset_states_horizontal (support_funcs.cpp:88-138): per row i = 1..N
  // the wetting loop along j, then the drying loop along j. The reference
  // runs one thread per row; rows are independent (a row's loops read and
  // write the mask, depths and levels of its own cells only), so they are
  // taken one after another here.
  void reset_states_horizontal() {
    const int off = W;
    for (int i = 1; i <= N; ++i) {
      for (int j = 2; j <= M; ++j) {
        if (tz[i * off + j] > z[i * off + j]) {
          if (khouot[i * off + j - 1] == 1) {
            tz[i * off + j - 1] = tz[i * off + j];
            Hmoi[i * off + j - 1] = htaiz[i * off + j - 1] + tz[i * off + j];
            khouot[i * off + j - 1] = 0;
            FS[i * off + j - 1] = FS[i * off + j];
          }
          if (khouot[i * off + j + 1] == 1) {
            tz[i * off + j + 1] = tz[i * off + j];
            Hmoi[i * off + j + 1] = htaiz[i * off + j + 1] + tz[i * off + j];
            khouot[i * off + j + 1] = 0;
            FS[i * off + j + 1] = FS[i * off + j];
          }
        }
      }
      for (int j = 2; j <= M; ++j) {
        if ((khouot[i * off + j] == 0) && (Hmoi[i * off + j] <= c.H_TINH)) {
          tu[(i - 1) * off + j] = 0;
          tu[i * off + j] = 0;
          tv[i * off + j - 1] = 0;
          tv[i * off + j] = 0;
          khouot[i * off + j] = 1;
          FS[i * off + j] = 0;
        }
      }
    }
  }

  // --------------------------------------------------------- sediment
  // Find_VTH, sediment_transport.cpp:575-602.
  void find_vth(int i_hi) {
    for (int i = 2; i <= i_hi; ++i)
      for (int j = 2; j <= M; ++j) {
        const int p = id(i, j);
        if ((htaiz[p] > c.NANGDAY) && (Hmoi[p] > c.H_TINH)) {
          const double ut = (tu[p] + tu[p - W]) * 0.5;
          const double vt = (tv[p] + tv[p - 1]) * 0.5;
          VTH[p] = std::sqrt(ut * ut + vt * vt);
        } else {
          VTH[p] = 0;
        }
      }
  }
  // hesoK, sediment_transport.cpp:539-573.
  void heso_k(int i_hi) {
    const double sg = std::sqrt(c.g);
    for (int i = 1; i <= i_hi; ++i)
      for (int j = 1; j <= M; ++j) {
        const int p = id(i, j);
        if (Htdu[p] > 0) {
          const double Cz = 18 * std::log(12 * Htdu[p] / c.Ks);
          double k = 5.93 * sg * (h[p - 1] + h[p]) * 0.25 * std::fabs(tu[p]) / Cz;
          Kx[p] = std::min(100.0, std::max(5.0, k));
        }
        if (Htdv[p] > 0) {
          const double Cz = 18 * std::log(12 * Htdv[p] / c.Ks);
          double k = 5.93 * sg * (h[p - W] + h[p]) * 0.25 * std::fabs(tv[p]) / Cz;
          Ky[p] = std::min(100.0, std::max(5.0, k));
        }
      }
  }
  // source_chs, sediment_transport.cpp:11-38.
  double source_chs(double wsm, double Zf, double fs, double fw, double vth, double h_moi) const {
    double toee = c.Toe, todd = c.Tod, S = 0;
    const double tob = c.ro * fw * (vth * vth);
    if (h_moi > c.ghtoe) toee = toee * (1 + c.hstoe * ((h_moi - c.ghtoe)));
    if (tob > toee) {
      S = c.Mbochat / c.ros * (tob - toee) / toee;
    } else if (tob < todd) {
      const double Pd = 1 - (tob / todd);
      const double beta = 1 + (Zf / (1.25 + 4.75 * std::pow(Pd, 2.5)));
      const double Cb = beta * fs;
      S = -wsm * Cb * Pd;
    }
    return S;
  }
  // source_nchs, sediment_transport.cpp:41-49.
  double source_nchs(double wsm, double Zf, double Uf, double h_moi, double fs) const {
    const double gamac = 0.434 + 5.975 * Zf + 2.888 * Zf * Zf;
    const double Tx = std::max(0.0, (Uf * Uf - c.Ufr * c.Ufr) / (c.Ufr * c.Ufr));
    const double Cac = 0.015 * c.dm * std::pow(Tx, 1.5) * std::pow(c.Dxr, (-0.3)) / (0.05 * h_moi);
    return wsm * (Cac - gamac * fs);
  }

  // Coefficients of one cell of a concentration sweep. xdir: the i-sweep
  // (_FSj_calculate__mactrix_coeff, sediment_transport.cpp:204-313) else the
  // j-sweep (_FSi_calculate__mactrix_coeff, :51-164).
  void fs_cell(bool xdir, int i, int j, double tt, double& A, double& B, double& C,
               double& D) const {
    const int pos = id(i, j);
    const double Ks = c.Ks, g = c.g, wss = c.wss, dY = c.dY, dX = c.dX, dT = c.dT,
                 H_TINH = c.H_TINH;
    const double cc = 18 * std::log(12 * Hmoi[pos] / Ks);
    const double Uf = std::sqrt(g) * std::fabs(VTH[pos]) / cc;
    const double wsm = wss * std::pow((1 - FS[pos]), 4);
    double Zf = 0, S;
    double gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;  // before Zf in the i-sweep (:247)
    if (FS[pos] > 0.00001) Zf = wsm / (0.4 * (Uf + 2 * wsm));
    if (o.ketdinh)
      S = source_chs(wsm, Zf, FS[pos], Fw[pos], VTH[pos], Hmoi[pos]);
    else
      S = source_nchs(wsm, Zf, Uf, Hmoi[pos], FS[pos]);
    if (tt < o.bed_change_start) S = 0;
    const int w = W;
    double p = 0, q = 0;
    if (xdir) {
      A = -gamav * 0.5 * (tu[pos] + tu[pos - w]) / (dX * 2) -
          Htdu[pos - w] * Kx[pos - w] / (Hmoi[pos] * (dX * dX));
      C = gamav * 0.5 * (tu[pos] + tu[pos - w]) / (dX * 2) -
          Htdu[pos] * Kx[pos] / (Hmoi[pos] * (dX * dX));
      B = 2.0 / dT + (Htdu[pos] * Kx[pos] + Htdu[pos - w] * Kx[pos - w]) / (Hmoi[pos] * (dX * dX));
      if ((Hmoi[pos - 1] > H_TINH) && (Hmoi[pos + 2] > H_TINH)) p = (FS[pos + 1] - FS[pos]);
      if ((Hmoi[pos - 2] > H_TINH) && (Hmoi[pos + 1] > H_TINH)) q = (FS[pos] - FS[pos - 1]);
      p = (1 / (Hmoi[pos] * (dY * dY))) * (Htdv[pos] * Ky[pos] * p - Htdv[pos - 1] * Ky[pos - 1] * q);
      if ((Hmoi[pos - 2] > H_TINH) && (Hmoi[pos + 2] > H_TINH)) {
        q = (FS[pos + 1] - FS[pos - 1]) / (dY * 2);
        q = (tv[pos] + tv[pos - 1]) * 0.5 * q * gamav;
      } else {
        q = 0;
      }
    } else {
      gamav = 0.98 - 0.198 * Zf + 0.032 * Zf * Zf;  // after Zf in the j-sweep (:109)
      A = -gamav * 0.5 * (tv[pos - 1] + tv[pos]) / (dY * 2) -
          Htdv[pos - 1] * Ky[pos - 1] / (Hmoi[pos] * (dY * dY));
      C = gamav * 0.5 * (tv[pos - 1] + tv[pos]) / (dY * 2) -
          Htdv[pos] * Ky[pos] / (Hmoi[pos] * (dY * dY));
      B = 2.0 / dT + (Htdv[pos] * Ky[pos] + Htdv[pos - 1] * Ky[pos - 1]) / (Hmoi[pos] * (dY * dY));
      if ((Hmoi[pos + 2 * w] > H_TINH) && (Hmoi[pos - w] > H_TINH)) p = (FS[pos + w] - FS[pos]);
      if (Hmoi[pos - 2 * w] > H_TINH && Hmoi[pos + w] > H_TINH) q = (FS[pos] - FS[pos - w]);
      p = (1 / (Hmoi[pos] * (dX * dX))) * (Htdu[pos] * Kx[pos] * p - Htdu[pos - w] * Kx[pos - w] * q);
      if (Hmoi[pos + 2 * w] > H_TINH && Hmoi[pos - 2 * w] > H_TINH) {
        q = (FS[pos + w] - FS[pos - w]) / (dX * 2);
        q = (tu[pos] + tu[pos - w]) * 0.5 * q * gamav;
      } else {
        q = 0;
      }
    }
    D = FS[pos] / (dT * 0.5) - q + p + (S / Hmoi[pos]);
  }

  // Concentration i-sweep of column j (Scan_FSj + tridiagSolver +
  // FSj_extract_solution, engine.cpp:156-167; sediment_transport.cpp:204-349).
  void fsj_column(LineBuf& L, int j, double tt) {
    const int w = W;
    for (int k = 0; k < mocj[j]; ++k) {
      const int first = dauj[j * SEG + k], last = cuoij[j * SEG + k];
      if (last < first + 2) continue;  // no interior row: nothing extracted
      bool br1, br2;
      ends_u(j, first, last, br1, br2);
      for (int i = first + 1; i <= last - 1; ++i) {
        double A, B, C, D;
        fs_cell(true, i, j, tt, A, B, C, D);
        if (i == first + 1) {
          if ((br1) || (tu[first * w + j] == 0))
            B += A;
          else
            D -= A * FS[first * w + j];
        }
        if (i == last - 1) {
          if ((br2) && (tu[last * w + j] == 0))
            B += C;
          else
            D -= C * FS[last * w + j];
        }
        L.AA[i] = A;
        L.BB[i] = B;
        L.CC[i] = C;
        L.DD[i] = D;
      }
      const int sn = last - first - 2, pos = first + 1;
      thomas(sn, &L.AA[pos], &L.BB[pos], &L.CC[pos], &L.DD[pos], &L.x[pos], L.Ap, L.Bp);
      for (int i = first + 1; i <= last - 1; ++i) {
        const int p = i * w + j;
        tFS[p] = L.x[i];
        if (L.x[i] < 0) tFS[p] = c.NDnen;
        if (i == first + 1)
          tFS[first * w + j] = ((br1) || (tu[p - w] == 0)) ? tFS[p] : FS[first * w + j];
        if (i == last - 1)
          tFS[last * w + j] = ((br2) || (tu[p + w] == 0)) ? tFS[p] : FS[last * w + j];
      }
    }
  }

  // Concentration j-sweep of row i (Scan_FSi + tridiagSolver +
  // FSi_extract_solution, engine.cpp:267-279; sediment_transport.cpp:51-201).
  void fsi_row(LineBuf& L, int i, double tt) {
    const int w = W;
    for (int k = 0; k < moci[i]; ++k) {
      const int first = daui[i * SEG + k], last = cuoii[i * SEG + k];
      if (last < first + 2) continue;
      bool br1, br2;
      ends_v(i, first, last, br1, br2);
      for (int j = first + 1; j <= last - 1; ++j) {
        double A, B, C, D;
        fs_cell(false, i, j, tt, A, B, C, D);
        if (j == first + 1) {
          if ((br1) || (tv[i * w + first] == 0))
            B = B + A;
          else
            D = D - A * FS[i * w + first];
        }
        if (j == last - 1) {
          if ((br2) || (tv[i * w + last] == 0))
            B = B + C;
          else
            D = D - C * FS[i * w + last];
        }
        L.AA[j] = A;
        L.BB[j] = B;
        L.CC[j] = C;
        L.DD[j] = D;
      }
      const int sn = last - first - 2, pos = first + 1;
      thomas(sn, &L.AA[pos], &L.BB[pos], &L.CC[pos], &L.DD[pos], &L.x[pos], L.Ap, L.Bp);
      for (int j = first + 1; j <= last - 1; ++j) {
        const int p = i * w + j;
        if (L.x[j] < 0) L.x[j] = c.NDnen;
        tFS[p] = L.x[j];
        if (j == first + 1)
          tFS[i * w + first] = ((br1) || (tv[i * w + first] == 0)) ? tFS[p] : FS[i * w + first];
        if (j == last - 1)
          tFS[i * w + last] = ((br2) || (tv[i * w + last] == 0)) ? tFS[p] : FS[i * w + last];
      }
    }
  }

  // ------------------------------------------------------ bed change
  // Calculate_Qb (sediment_transport.cpp:352-434) and _bed_load / BedLoad
  // (:436-537, :664-673). The reference never launches them (its call is
  // commented out, engine.cpp:290-293); its code is read as intended where it
  // cannot be meant literally: the flux is computed where the speed is not
  // zero (:385 tests !VTH and then divides by VTH), Toee starts from the
  // coefficient Toe (:359 reads a shared copy before it is assigned), the
  // corner copies take both components under their condition (:410-419
  // lack braces), and the downwind test reads t_u[pos] > 0 (:479 indexes
  // t_u with a boolean).
  void calc_qb() {
    const int w = W;
    const double kq = 0.053 * std::sqrt((c.Sx - 1) * c.g) * std::pow(c.dm, 1.5);
    const double dxr = std::pow(c.Dxr, -0.3);
    for (int i = 2; i <= N; ++i)
      for (int j = 2; j <= M; ++j) {
        const int pos = id(i, j);
        double qx = 0, qy = 0;
        if (VTH[pos] != 0 && khouot[pos] == 0) {
          double Toee = c.Toe, Tx = 0;
          const double Tob = c.ro * Fw[pos] * (VTH[pos] * VTH[pos]);
          if (Hmoi[pos] > c.ghtoe) Toee = c.Toe * (1 + c.hstoe * ((Hmoi[pos] - c.ghtoe)));
          if (Tob > Toee) Tx = Tob / Toee - 1;
          const double base = kq * std::pow(Tx, 2.1) * dxr;
          qx = base * (tu[pos] + tu[pos - w]) * 0.5 / VTH[pos];
          qy = base * (tv[pos] + tv[pos - 1]) * 0.5 / VTH[pos];
        }
        Qbx[pos] = qx;
        Qby[pos] = qy;
      }
    // margins copy the nearest interior value (:402-431)
    for (int j = 2; j <= M; ++j) {
      Qbx[id(1, j)] = Qbx[id(2, j)];
      Qby[id(1, j)] = Qby[id(2, j)];
      Qbx[id(N + 1, j)] = Qbx[id(N, j)];
      Qby[id(N + 1, j)] = Qby[id(N, j)];
    }
    for (int i = 2; i <= N; ++i) {
      Qbx[id(i, 1)] = Qbx[id(i, 2)];
      Qby[id(i, 1)] = Qby[id(i, 2)];
      Qbx[id(i, M + 1)] = Qbx[id(i, M)];
      Qby[id(i, M + 1)] = Qby[id(i, M)];
    }
    const int corner[4][4] = {{1, 1, 2, 2}, {N + 1, 1, N, 2}, {1, M + 1, 2, M}, {N + 1, M + 1, N, M}};
    for (const auto& k : corner) {
      Qbx[id(k[0], k[1])] = Qbx[id(k[2], k[3])];
      Qby[id(k[0], k[1])] = Qby[id(k[2], k[3])];
    }
  }

  // _bed_load for rows 3..N-2 (BedLoad's launch with the j-sweep's range,
  // engine.cpp:292), cells of the row's wet segments of at least 3 cells.
  void bed_load() {
    const int w = W;
    const double dX = c.dX, dY = c.dY;
    for (int i = 3; i < N - 1; ++i)
      for (int k = 0; k < moci[i]; ++k) {
        const int first = daui[i * SEG + k], last = cuoii[i * SEG + k];
        if (last - first < 2) continue;
        for (int j = first; j <= last; ++j) {
          const int pos = id(i, j);
          double p = 0, q = 0;
          if (khouot[pos - w] == 1) {
            if (tu[pos] < 0) p = (-3 * Qbx[pos] + 4 * Qbx[pos + w] - Qbx[pos + 2 * w]) / (dX * 2);
          } else {
            if (khouot[pos + w] == 1) {
              if (tu[pos] > 0) p = (3 * Qbx[pos] - 4 * Qbx[pos - w] + Qbx[pos - 2 * w]) / (dX * 2);
            } else {
              p = (Qbx[pos + w] - Qbx[pos - w]) / (dX * 2);
            }
          }
          if (khouot[pos - 1] == 1) {
            if (tv[pos] < 0) q = (-3 * Qby[pos] + 4 * Qby[pos + 1] - Qby[pos + 2]) / (dY * 2);
          } else {
            if (khouot[pos + 1] == 1) {
              if (tv[pos] > 0) q = (3 * Qby[pos] - 4 * Qby[pos - 1] + Qby[pos - 2]) / (dY * 2);
            } else {
              q = (Qby[pos + 1] - Qby[pos - 1]) / (dY * 2);
            }
          }
          double tH = p + q;
          p = FS[pos + w] - FS[pos];
          if ((khouot[pos + 2 * w] == 1 || khouot[pos - w] == 1) && (i < N)) p = 0;
          q = FS[pos] - FS[pos - w];
          if ((i > 2) && (khouot[pos - 2 * w] == 1 || khouot[pos + w] == 1)) q = 0;
          p = 1 / (dX * dX) * (Htdu[pos] * Kx[pos] * p - Htdu[pos - w] * Kx[pos - w] * q);
          tH = tH + p;
          p = FS[pos + 1] - FS[pos];
          if (((last < M) && (khouot[pos - 1] == 1 || khouot[pos + 2] == 1)) ||
              (last == M && (khouot[pos - 1] == 1)))
            p = 0;
          q = FS[pos] - FS[pos - 1];
          if (((first > 2) && (khouot[pos - 2] == 1 || khouot[pos + 1] == 1)) ||
              (first == 2 && khouot[pos + 1] == 1))
            q = 0;
          p = 1 / ((dY * dY)) * (Htdv[pos] * Ky[pos] * p - Htdv[pos - 1] * Ky[pos - 1] * q);
          tH = tH + p;
          const double cc = 18 * std::log(12 * Hmoi[pos] / c.Ks);
          const double Uf = std::sqrt(c.g) * std::fabs(VTH[pos]) / cc;
          const double wsm = c.wss * std::pow((1 - FS[pos]), 4);
          double Zf = 0;
          if (FS[pos] > 0.0) Zf = wsm / (0.4 * (Uf + 2 * wsm));
          const double S = o.ketdinh ? source_chs(wsm, Zf, FS[pos], Fw[pos], VTH[pos], Hmoi[pos])
                                     : source_nchs(wsm, Zf, Uf, Hmoi[pos], FS[pos]);
          dH[pos] += c.dT / (1 - c.Dorong) * (S + tH);
        }
      }
  }

  // Update_FS, sediment_transport.cpp:654-663.
  void update_fs() {
    for (int i = 1; i <= N; ++i)
      for (int j = 1; j <= M; ++j) FS[id(i, j)] = tFS[id(i, j)];
  }

  // --------------------------------------------------------- driver
  std::vector<LineBuf> bufs;
  std::vector<double> tmpbuf;

  LineBuf& buf(int tid) { return bufs[tid]; }

  template <class F>
  void for_lines(int lo, int hi_incl, F&& f) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (int k = lo; k <= hi_incl; ++k) {
#ifdef _OPENMP
      const int tid = omp_get_thread_num();
#else
      const int tid = 0;
#endif
      f(buf(tid), k);
    }
  }

  void alloc_bufs() {
    int nt = 1;
#ifdef _OPENMP
    nt = std::max(1, nthreads);
#endif
    bufs.resize(nt);
    const int nmax = std::max(M, N) + 4;
    for (auto& b : bufs) b.size(nmax + 2, 2 * nmax + 4);
  }

  // The same step split into its operations, for inspecting intermediate
  // states: runs operations [0, nops) of one step and returns how many exist.
  int step_ops(int nops) {
    int k = 0;
    auto op = [&](auto&& f) {
      if (k < nops) f();
      ++k;
    };
    op([&] { t += 0.5 * c.dT; boundary(t); });
    op([&] { for_lines(2, M, [&](LineBuf& L, int j) { uz_column(L, j); }); });
    op([&] { normalize(true, tmpbuf); });
    op([&] { solve_v(); });
    op([&] { margin_v(); });
    op([&] { normalize(false, tmpbuf); });
    op([&] { update_h_moi(); update_uvz(); find_limits(); htuongdoi(); });
    op([&] { t += c.dT * 0.5; boundary(t); });
    op([&] { for_lines(2, N, [&](LineBuf& L, int i) { vz_row(L, i); }); });
    op([&] { normalize(false, tmpbuf); });
    op([&] { solve_u(); });
    op([&] { margin_u(); });
    op([&] { normalize(true, tmpbuf); });
    op([&] { update_h_moi(); });
    op([&] { reset_states_vertical(); });
    op([&] { update_uvz(); find_limits(); htuongdoi(); });
    return k;
  }

  // One full step: the body of the while-loop of Hydraulic_Calculation,
  // engine.cpp:65-295.
  void step() {
    // ---- first half: UZ sweep, explicit v (engine.cpp:66-170); in channel
    // mode with kenhhepd the sweep takes columns 3..M-1 (engine.cpp:77-80)
    t += 0.5 * c.dT;
    update_boundary(t);
    const bool narrow_x = channel() && o.kenhhepd;
    for_lines(narrow_x ? 3 : 2, narrow_x ? M - 1 : M, [&](LineBuf& L, int j) { uz_column(L, j); });
    normalize(true, tmpbuf);
    solve_v();
    margin_v();
    normalize(false, tmpbuf);
    update_h_moi();
    // wetting/drying along rows, where Reset_states_vertical has its place
    // in the second half (the reference never launches it)
    if (o.reset_horizontal) reset_states_horizontal();
    update_uvz();
    find_limits();
    htuongdoi();
    if (t >= o.sediment_start) {
      find_vth(N);
      heso_k(N);
      const double tt = t;
      for_lines(3, M - 1, [&](LineBuf& L, int j) { fsj_column(L, j, tt); });
      update_fs();
    }
    // ---- second half: VZ sweep, explicit u, wet/dry (engine.cpp:176-282);
    // rows 3..N with kenhhepng in channel mode (engine.cpp:190-193)
    t += c.dT * 0.5;
    update_boundary(t);
    const bool narrow_y = channel() && o.kenhhepng;
    for_lines(narrow_y ? 3 : 2, N, [&](LineBuf& L, int i) { vz_row(L, i); });
    normalize(false, tmpbuf);
    solve_u();
    margin_u();
    normalize(true, tmpbuf);
    update_h_moi();
    reset_states_vertical();
    update_uvz();
    find_limits();
    htuongdoi();
    if (t >= o.sediment_start) {
      find_vth(N - 1);
      heso_k(N - 1);
      const double tt = t;
      for_lines(3, N - 1, [&](LineBuf& L, int i) { fsi_row(L, i, tt); });
      update_fs();
      // the bed change once per step after the j-sweep (engine.cpp:290-293)
      if (o.bed_change && t >= o.bed_change_start) {
        calc_qb();
        bed_load();
        if (o.bed_feedback) bed_feedback();
      }
    }
  }
};

void set_err(const char* m) { g_err = m; }

}  // namespace

struct OracleSim {
  Sim s;
};

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

OracleSim* oracle_create(const HydistScenario* sc, const HydistParams* p,
                         const HydistOptions* o, int nthreads) {
  if (!sc || !p || !o) {
    set_err("null argument");
    return nullptr;
  }
  if (sc->M < 4 || sc->N < 4 || sc->total_time < 2 || !sc->h || !sc->hsnham || !sc->visco ||
      !sc->Fw || !sc->boundary_type || sc->n_boundary_type < 4 * SEG) {
    set_err("bad scenario");
    return nullptr;
  }
  auto* os = new OracleSim();
  Sim& s = os->s;
  s.M = sc->M;
  s.N = sc->N;
  s.W = s.M + 3;
  s.H = s.N + 3;
  s.T = sc->total_time;
  s.nthreads = nthreads > 0 ? nthreads : 1;
  derive(*p, s.c);
  s.o = *o;
  s.t = o->t_start;
  const size_t n = (size_t)s.W * s.H;
  s.h.assign(sc->h, sc->h + n);
  s.hsnham.assign(sc->hsnham, sc->hsnham + n);
  s.visco.assign(sc->visco, sc->visco + n);
  s.Fw.assign(sc->Fw, sc->Fw + n);
  const double* bcs[4] = {sc->bc_up, sc->bc_down, sc->bc_left, sc->bc_right};
  const double* ccs[4] = {sc->CC_up, sc->CC_down, sc->CC_left, sc->CC_right};
  for (int k = 0; k < 4; ++k) {
    s.bc[k].assign(s.T, 0.0);
    s.CC[k].assign(s.T, 0.0);
    if (bcs[k]) std::copy(bcs[k], bcs[k] + s.T, s.bc[k].begin());
    if (ccs[k]) std::copy(ccs[k], ccs[k] + s.T, s.CC[k].begin());
    s.bienQ[k] = sc->bienQ[k];
  }
  s.btype.assign(sc->boundary_type, sc->boundary_type + 4 * SEG);
  for (auto* vp : {&s.u, &s.v, &s.z, &s.tu, &s.tv, &s.tz, &s.Hmoi, &s.htaiz, &s.htaiz_bd,
                   &s.Htdu, &s.Htdv, &s.Kx1, &s.Ky1, &s.Tsxw, &s.Tsyw, &s.FS, &s.tFS, &s.VTH,
                   &s.Kx, &s.Ky, &s.dH, &s.Qbx, &s.Qby})
    vp->assign(n, 0.0);
  s.khouot.assign(n, 0);
  s.ubt.assign(s.M + 3, 0.0);
  s.ubp.assign(s.M + 3, 0.0);
  s.vbt.assign(s.N + 3, 0.0);
  s.vbd.assign(s.N + 3, 0.0);
  s.hi.assign(2 * (s.M + s.N + 6), 0.0);
  s.daui.assign((s.N + 3) * SEG, 0);
  s.cuoii.assign((s.N + 3) * SEG, 0);
  s.moci.assign(s.N + 3, 0);
  s.dauj.assign((s.M + 3) * SEG, 0);
  s.cuoij.assign((s.M + 3) * SEG, 0);
  s.mocj.assign(s.M + 3, 0);
  if (sc->FS0) {
    s.FS.assign(sc->FS0, sc->FS0 + n);
    s.tFS = s.FS;
  }
  if (sc->z0) {
    s.z.assign(sc->z0, sc->z0 + n);
    s.tz = s.z;
  }
  s.alloc_bufs();
  // set-up sequence of main.cpp:262-298
  s.onetime_init();
  s.find_limits();
  s.htuongdoi();
  s.preprocess_data();
  if (o->bed_feedback) s.keep_initial_bed();
  if (s.seg_overflow) {
    set_err("more than 20 wet segments in a line");
    delete os;
    return nullptr;
  }
  return os;
}

void oracle_destroy(OracleSim* os) { delete os; }

void oracle_set_race_mode(OracleSim* os, int race_new) { os->s.race_new = race_new; }

int oracle_step(OracleSim* os, int nsteps) {
  for (int k = 0; k < nsteps; ++k) {
    os->s.step();
    if (os->s.seg_overflow) {
      set_err("more than 20 wet segments in a line");
      return HYDIST_ERR_SEGMENTS;
    }
  }
  return HYDIST_OK;
}

double oracle_time(OracleSim* os) { return os->s.t; }

void oracle_set_time(OracleSim* os, double t) { os->s.t = t; }

// Rebuild the wet-segment tables from the mask (after oracle_set of the
// mask); HYDIST_ERR_SEGMENTS if a line has more than 20 wet segments.
int oracle_rescan_segments(OracleSim* os) {
  os->s.seg_overflow = false;
  os->s.rescan_segments();
  if (os->s.seg_overflow) {
    set_err("more than 20 wet segments in a line");
    return HYDIST_ERR_SEGMENTS;
  }
  return HYDIST_OK;
}

// Debug: run the first nops operations of one hydraulic step (no sediment).
int oracle_step_ops(OracleSim* os, int nops) { return os->s.step_ops(nops); }

int oracle_get(OracleSim* os, int field, void* out) {
  Sim& s = os->s;
  const size_t n = (size_t)s.W * s.H;
  if (field == HYDIST_FIELD_KHOUOT) {
    std::memcpy(out, s.khouot.data(), n * sizeof(int));
    return HYDIST_OK;
  }
  auto* f = s.field(field);
  if (!f) return HYDIST_ERR_ARG;
  std::memcpy(out, f->data(), n * sizeof(double));
  return HYDIST_OK;
}

int oracle_set(OracleSim* os, int field, const void* in) {
  Sim& s = os->s;
  const size_t n = (size_t)s.W * s.H;
  if (field == HYDIST_FIELD_KHOUOT) {
    std::memcpy(s.khouot.data(), in, n * sizeof(int));
    return HYDIST_OK;
  }
  auto* f = s.field(field);
  if (!f) return HYDIST_ERR_ARG;
  std::memcpy(f->data(), in, n * sizeof(double));
  return HYDIST_OK;
}

// Segment tables: kind 0 = rows (daui/cuoii/moci), 1 = columns.
int oracle_get_segments(OracleSim* os, int kind, int* dau, int* cuoi, int* moc) {
  Sim& s = os->s;
  if (kind == 0) {
    std::copy(s.daui.begin(), s.daui.end(), dau);
    std::copy(s.cuoii.begin(), s.cuoii.end(), cuoi);
    std::copy(s.moci.begin(), s.moci.end(), moc);
  } else {
    std::copy(s.dauj.begin(), s.dauj.end(), dau);
    std::copy(s.cuoij.begin(), s.cuoij.end(), cuoi);
    std::copy(s.mocj.begin(), s.mocj.end(), moc);
  }
  return HYDIST_OK;
}

// Boundary vectors: ubt, ubp (M+3 each), vbt, vbd (N+3 each), hi (2(M+N+6)).
int oracle_get_boundary(OracleSim* os, double* ubt, double* ubp, double* vbt, double* vbd,
                        double* hi, double* hmax4) {
  Sim& s = os->s;
  std::copy(s.ubt.begin(), s.ubt.end(), ubt);
  std::copy(s.ubp.begin(), s.ubp.end(), ubp);
  std::copy(s.vbt.begin(), s.vbt.end(), vbt);
  std::copy(s.vbd.begin(), s.vbd.end(), vbd);
  std::copy(s.hi.begin(), s.hi.end(), hi);
  hmax4[0] = s.hmax_u;
  hmax4[1] = s.hmax_d;
  hmax4[2] = s.hmax_l;
  hmax4[3] = s.hmax_r;
  return HYDIST_OK;
}

// Plain Thomas on one system (tridiag, UVZSolver_multithread.cpp:19-43):
// n = system size, dl[0] and du[n-1] ignored.
int oracle_thomas(int n, const double* dl, const double* d, const double* du, const double* b,
                  double* x) {
  if (n <= 0) return HYDIST_ERR_ARG;
  std::vector<double> Ap, Bp;
  Sim::thomas(n - 1, dl, d, du, b, x, Ap, Bp);
  return HYDIST_OK;
}

// Batched plain Thomas over packed systems; OpenMP over systems.
int oracle_thomas_batched(const double* dl, const double* d, const double* du, const double* b,
                          double* x, const int* offsets, const int* lengths, int nsys,
                          int nthreads) {
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
#endif
  {
    std::vector<double> Ap, Bp;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
    for (int s = 0; s < nsys; ++s) {
      const int o = offsets[s], n = lengths[s];
      if (n > 0) Sim::thomas(n - 1, dl + o, d + o, du + o, b + o, x + o, Ap, Bp);
    }
  }
  return HYDIST_OK;
}

}  // extern "C"
