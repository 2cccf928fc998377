// compat.cu -- the reference's time-step entry points (engine.cpp) with
// their C++ signatures, on top of the C ABI.
//
// Hydraulic_Calculation (engine.cpp:41-296) receives device pointers to the
// reference's structs and a host copy of Argument_Pointers whose members are
// the caller's device arrays. It adopts those arrays with
// hydist_create_external (no copy), runs the time loop by half-steps and
// calls the reference's result writers at the reference's times:
//   - after half-step A when t is an integer multiple of ops.interval
//     (engine.cpp:143-144; u, v, z after its commit);
//   - in half-step B at such t before update_uvz (engine.cpp:237-238); no
//     kernel of half-step B before update_uvz writes u, v or z, so these are
//     the values after half-step A, written before half-step B runs;
//   - save_FS after half-step B's concentration sweep when t is a multiple
//     of 360 s (engine.cpp:280-284, ros = 2000 as there).
// The writers live in the reference's loader.cpp; they are weak references
// here, so the library links without them and a program that links
// loader.cpp gets its outputs.
#include <cassert>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>

#include "../../include/hydist_capi.h"
#include "../../include/hydist_compat.h"

void save_result(Argument_Pointers h_arg_pointer, int t) __attribute__((weak));
void save_FS(Argument_Pointers h_arg_pointer, int t, double ros) __attribute__((weak));

namespace {

[[noreturn]] void compat_fail(const char* what) {
  std::fprintf(stderr, "hydist: %s: %s\n", what, hydist_last_error());
  std::abort();
}

#define HC(call)                               \
  do {                                         \
    if ((call) != HYDIST_OK) compat_fail(#call); \
  } while (0)

#define CC(call)                                                                \
  do {                                                                          \
    cudaError_t e__ = (call);                                                   \
    if (e__ != cudaSuccess) {                                                   \
      std::fprintf(stderr, "hydist: %s: %s\n", #call, cudaGetErrorString(e__)); \
      std::abort();                                                             \
    }                                                                           \
  } while (0)

// Load_coeffs' inputs from the caller's Constant_Coeffs (the derived
// constants are recomputed from them by the library with the same formulas)
HydistParams params_of(const Constant_Coeffs& c, double dT, double NANGDAY) {
  HydistParams p;
  hydist_params_default(&p);
  p.dX = c.dX;
  p.dY = c.dY;
  p.dT = dT;
  p.NANGDAY = NANGDAY;
  p.H_TINH = c.H_TINH;
  p.heso = c.heso;
  p.mu_mn = c.mu_mn;
  p.NDnen = c.NDnen;
  p.Tod = c.Tod;
  p.Toe = c.Toe;
  p.hstoe = c.hstoe;
  p.ghtoe = c.ghtoe;
  p.Mbochat = c.Mbochat;
  p.ro = c.ro;
  p.ros = c.ros;
  p.dm = c.dm;
  p.d90 = c.d90;
  p.muy = c.muy;
  p.Dorong = c.Dorong;
  p.Sx = c.Sx;
  p.CORIOLIS_FORCE = c.CORIOLIS_FORCE;
  p.g = c.g;
  p.Wind = c.Wind;
  p.huonggio = c.huonggio;
  p.wss = c.wss;
  p.Ks = c.Ks;
  return p;
}

HydistExternal external_of(const Argument_Pointers& a, int total_time, const int bienQ[4]) {
  HydistExternal e{};
  e.M = a.M;
  e.N = a.N;
  e.total_time = total_time;
  for (int k = 0; k < 4; ++k) e.bienQ[k] = bienQ[k];
  e.h = a.h;
  e.hsnham = a.hsnham;
  e.visco = a.VISCOIDX;
  e.Fw = a.Fw;
  e.htaiz = a.htaiz;
  e.htaiz_bd = a.htaiz_bd;
  e.Kx1 = a.Kx1;
  e.Ky1 = a.Ky1;
  e.Tsxw = a.Tsxw;
  e.Tsyw = a.Tsyw;
  e.bc_up = a.bc_up;
  e.bc_down = a.bc_down;
  e.bc_left = a.bc_left;
  e.bc_right = a.bc_right;
  e.CC_up = a.CC_u;
  e.CC_down = a.CC_d;
  e.CC_left = a.CC_l;
  e.CC_right = a.CC_r;
  e.boundary_type = a.boundary_type;
  e.u = a.u;
  e.v = a.v;
  e.z = a.z;
  e.t_u = a.t_u;
  e.t_v = a.t_v;
  e.t_z = a.t_z;
  e.H_moi = a.H_moi;
  e.Htdu = a.Htdu;
  e.Htdv = a.Htdv;
  e.FS = a.FS;
  e.tFS = a.tFS;
  e.VTH = a.VTH;
  e.Kx = a.Kx;
  e.Ky = a.Ky;
  e.dH = a.dH;
  e.Qbx = a.Qbx;
  e.Qby = a.Qby;
  e.khouot = a.khouot;
  e.daui = a.daui;
  e.cuoii = a.cuoii;
  e.moci = a.moci;
  e.dauj = a.dauj;
  e.cuoij = a.cuoij;
  e.mocj = a.mocj;
  e.ubt = a.ubt;
  e.ubp = a.ubp;
  e.vbt = a.vbt;
  e.vbd = a.vbd;
  return e;
}

// A handle over the caller's arrays; the Options fields that the time step
// reads become HydistOptions.
HydistHandle* adopt(const Argument_Pointers& a, const Constant_Coeffs& c, double dT,
                    double NANGDAY, int total_time, double t_start, double sediment_start,
                    double bed_change_start, bool ketdinh, bool kenhhepd = false,
                    bool kenhhepng = false) {
  // update_uvz's coefficients (support_funcs.cpp:745-758); Load_coeffs sets
  // both to 0 (loader.cpp:18-19) whatever the options
  if (c.kenhhepd != 0 || c.kenhhepng != 0)
    compat_fail("Constant_Coeffs kenhhepd/kenhhepng other than 0 are not supported");
  int bienQ[4] = {0, 0, 0, 0};
  CC(cudaMemcpy(bienQ, a.bienQ, sizeof(bienQ), cudaMemcpyDeviceToHost));
  const HydistExternal e = external_of(a, total_time, bienQ);
  const HydistParams p = params_of(c, dT, NANGDAY);
  HydistOptions o;
  hydist_options_default(&o);
  o.t_start = t_start;
  o.sediment_start = sediment_start;
  o.bed_change_start = bed_change_start;
  o.ketdinh = ketdinh ? 1 : 0;
  o.kenhhepd = kenhhepd ? 1 : 0;
  o.kenhhepng = kenhhepng ? 1 : 0;
  HydistHandle* h = nullptr;
  HC(hydist_create_external(&e, &p, &o, -1, &h));
  return h;
}

bool due(double t, int every) { return every > 0 && ((int)t % every == 0) && (t - (int)t == 0); }

// update_boundary_at_t may be called on its own many times: one handle per
// device struct, kept for the process lifetime (the reference never frees
// its device arrays either).
std::mutex g_mu;
std::map<const Argument_Pointers*, HydistHandle*> g_boundary_handles;

}  // namespace

void synch_and_check() {
  cudaDeviceSynchronize();
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) std::fprintf(stderr, "error: %s\n", cudaGetErrorString(err));
  assert(err == cudaSuccess);
}

void update_boundary_at_t(int M, int N, float t, bool channel, int total_time,
                          Argument_Pointers* d_arg_ptr, Constant_Coeffs* coeffs) {
  (void)M;
  (void)N;
  if (channel) return;  // the reference's narrow-channel boundaries are disabled (engine.cpp:24-29)
  HydistHandle* h = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_boundary_handles.find(d_arg_ptr);
    if (it == g_boundary_handles.end()) {
      // previous work on the legacy stream must be done before the
      // library's stream reads the arrays
      CC(cudaDeviceSynchronize());
      Argument_Pointers a;
      Constant_Coeffs c;
      CC(cudaMemcpy(&a, d_arg_ptr, sizeof(a), cudaMemcpyDeviceToHost));
      CC(cudaMemcpy(&c, coeffs, sizeof(c), cudaMemcpyDeviceToHost));
      h = adopt(a, c, c.dT, c.NANGDAY, total_time, 0.0, 1e300, 1e300, true);
      g_boundary_handles[d_arg_ptr] = h;
    } else {
      h = it->second;
      CC(cudaDeviceSynchronize());
    }
  }
  HC(hydist_update_boundary(h, (double)t));
  HC(hydist_sync(h));
}

void Hydraulic_Calculation(double dT, double NANGDAY, Argument_Pointers* d_arg_ptr,
                           Array_Pointers* d_arr_ptr, Constant_Coeffs* coeffs,
                           Argument_Pointers h_arg_ptr, Options ops) {
  (void)d_arg_ptr;
  (void)d_arr_ptr;
  CC(cudaDeviceSynchronize());
  Constant_Coeffs c;
  CC(cudaMemcpy(&c, coeffs, sizeof(c), cudaMemcpyDeviceToHost));
  // the narrow-channel mode (ops.channel = kenhhepd xor kenhhepng) is the
  // handle's: no boundary update and the sweeps' index ranges of
  // engine.cpp:77-80, 190-193
  HydistHandle* h = adopt(h_arg_ptr, c, dT, NANGDAY, ops.total_time, ops.t_start,
                          ops.sediment_start, ops.bed_change_start, ops.ketdinh, ops.kenhhepd,
                          ops.kenhhepng);
  double t = ops.t_start;
  const int Tmax = (int)ops.Tmax;  // the reference compares with int(Tmax)
  while (t < Tmax) {
    t += 0.5 * dT;
    HC(hydist_half_step(h, 0));
    if (save_result && due(t, ops.interval)) {
      HC(hydist_sync(h));
      save_result(h_arg_ptr, (int)t);
    }
    t += dT * 0.5;
    if (save_result && due(t, ops.interval)) {
      HC(hydist_sync(h));
      save_result(h_arg_ptr, (int)t);
    }
    HC(hydist_half_step(h, 1));
    if (t >= ops.sediment_start && save_FS && due(t, 360)) {
      HC(hydist_sync(h));
      save_FS(h_arg_ptr, (int)t, 2000.0);
    }
  }
  HC(hydist_sync(h));
  HC(hydist_destroy(h));
}
