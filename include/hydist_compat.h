/*
 * hydist_compat.h -- C++ drop-in for the reference's time-step entry points.
 *
 * The structs below have the reference's member types and order (engine.h:
 * 16-89: Options, Constant_Coeffs, Argument_Pointers, Array_Pointers), so a
 * program written against the reference's engine.h -- its main.cpp and
 * loader.cpp included -- compiles and links against this library unchanged:
 * the functions declared here replace engine.cpp's Hydraulic_Calculation,
 * update_boundary_at_t and synch_and_check with the same signatures (C++
 * linkage). They run on the caller's device arrays in place through
 * hydist_create_external; Array_Pointers is accepted and not used (the
 * library's solver keeps its own, smaller scratch).
 *
 * A program that includes the reference's engine.h must not include this
 * header as well; the two declare the same types.
 */
#ifndef HYDIST_COMPAT_H
#define HYDIST_COMPAT_H

#include <cuda_runtime.h>

struct Options {
  double Tmax, t_start, sediment_start, bed_change_start;
  int interval;
  bool kenhhepd, kenhhepng;
  int M, N;
  bool ketdinh, channel, debug, plot;
  int total_time;
  Options(double Tmx, double ts, int itv, double sds, double bcs, bool cohesive, bool kenhng,
          bool kenhd, bool db, bool plt)
      : Tmax(Tmx), t_start(ts), sediment_start(sds), bed_change_start(bcs), interval(itv),
        kenhhepd(kenhd), kenhhepng(kenhng), M(0), N(0), ketdinh(cohesive),
        channel(kenhd ^ kenhng), debug(db), plot(plt), total_time(0) {}
};

struct Constant_Coeffs {
  double dX, dY, dT, dXbp, dYbp, dX2, dY2, dTchia2dX, dTchia2dY, HaiChiadT;
  double QuyDoiTime, QuyDoiPi;
  double NANGDAY, H_TINH, heso, mu_mn;
  double kenhhepng, kenhhepd;
  double Wind, huonggio, Zbandau;
  double NDnen, NDbphai, NDbtrai, NDbtren, NDbduoi;
  double Tod, Toe, hstoe, ghtoe, Mbochat;
  double ro, ros, dm, muy, d90, Dorong, Sx, sohn, soha, sohn1;
  double CORIOLIS_FORCE, g, Ks;
  double Windx, Windy, Ufr, Dxr, wss;
};

struct Argument_Pointers {
  int M, N;
  double hmax_u, hmax_d, hmax_l, hmax_r;
  int* bienQ;
  int *daui, *dauj, *cuoii, *cuoij, *moci, *mocj, *khouot, *boundary_type;
  double *h, *v, *u, *z, *t_u, *t_v, *t_z, *Htdu, *Htdv, *H_moi, *htaiz, *htaiz_bd;
  double *ubt, *ubp, *vbt, *vbd;
  double *hsnham, *VISCOIDX, *Kx1, *Ky1, *Tsyw, *Tsxw;
  double *bc_up, *bc_down, *bc_left, *bc_right;
  double* hi;
  double *FS, *tFS, *CC_u, *CC_d, *CC_l, *CC_r;
  double *VTH, *Kx, *Ky, *Fw;
  double *Qbx, *Qby;
  double* dH;
};

struct Array_Pointers {
  double *a1, *b1, *c1, *d1, *a2, *c2, *d2;
  double *f1, *f2, *f3, *f5;
  double *AA, *BB, *CC, *DD;
  double* x;
  double *Ap, *Bp, *ep;
  int* SN;
};

/* engine.cpp:22-36: the boundary update at time t (d_arg_ptr and coeffs are
 * device pointers to the structs, as the reference passes them). */
void update_boundary_at_t(int M, int N, float t, bool channel, int total_time,
                          Argument_Pointers* d_arg_ptr, Constant_Coeffs* coeffs);

/* engine.cpp:12-19: synchronise the device and assert on an error. */
void synch_and_check();

/* engine.cpp:41-296: the time loop from ops.t_start while t < (int)ops.Tmax,
 * in place on the caller's arrays. Writes results through the reference's
 * save_result / save_FS (loader.cpp:397-440) when the program links them,
 * at the same times and with the same fields as the reference. */
void Hydraulic_Calculation(double dT, double NANGDAY, Argument_Pointers* d_arg_ptr,
                           Array_Pointers* d_arr_ptr, Constant_Coeffs* coeffs,
                           Argument_Pointers h_arg_ptr, Options ops);

#endif
