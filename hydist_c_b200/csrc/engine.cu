// engine.cu -- host side of the B200 Hydist time step behind the C ABI.
//
// hydist_create  replaces main.cpp:138-304 (allocation loader.cpp:224-375,
//                Load_coeffs loader.cpp:4-87, set-up kernels)
// hydist_step    replaces the time loop of Hydraulic_Calculation
//                (engine.cpp:41-296); every launch goes to the handle's
//                stream, with no device-wide synchronisation between kernels
//                (the reference synchronises after each, engine.cpp:13-19)
// hydist_step_graph  the same step captured once into a CUDA graph per
//                sediment phase and replayed
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "hydro.cuh"

using namespace hyd;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& m) {
  g_err = m;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e__ = (call);                                                             \
    if (e__ != cudaSuccess)                                                               \
      return fail(e__ == cudaErrorMemoryAllocation ? HYDIST_ERR_OOM : HYDIST_ERR_CUDA,    \
                  std::string(#call) + ": " + cudaGetErrorString(e__));                   \
  } while (0)

const double kPI = 3.14159265358979323846;

void derive(const HydistParams& p, Coef& c) {
  // Load_coeffs, loader.cpp:4-87 (operator order kept)
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
  c.Ks = p.Ks >= 0 ? p.Ks : 2.5 * c.dm;
  c.Windx = 0.0013 * (0.00075 + 0.000067 * std::fabs(p.Wind)) * std::fabs(p.Wind) * p.Wind *
            std::cos(p.huonggio * (kPI / 180));
  c.Windy = 0.0013 * (0.00075 + 0.000067 * std::fabs(p.Wind)) * std::fabs(p.Wind) * p.Wind *
            std::sin(p.huonggio * (kPI / 180));
  c.Ufr = 0.25 * std::pow((c.Sx - 1) * c.g, 8.0 / 15.0) * std::pow(c.dm, 9.0 / 15.0) *
          std::pow(c.muy, -1.0 / 15.0);
  c.Dxr = c.dm * std::pow(c.g * (c.Sx - 1) / c.muy * c.muy, (1.0 / 3.0));
  c.wss = p.wss >= 0 ? p.wss
                     : 10 * c.muy / c.dm *
                           (std::sqrt(1 + 0.01 * (c.Sx - 1) * 9.81 * std::pow(c.dm, 3) /
                                              std::pow(c.muy, 2)) -
                            1);
  c.r_dX = 1.0 / c.dX;
  c.r_dY = 1.0 / c.dY;
  c.r_dX2 = 1.0 / c.dX2;
  c.r_dY2 = 1.0 / c.dY2;
  c.r_dXbp = 1.0 / c.dXbp;
  c.r_dYbp = 1.0 / c.dYbp;
  c.dT_dXbp = c.dT / c.dXbp;
  c.dT_dYbp = c.dT / c.dYbp;
  c.sqrt_g = std::sqrt(c.g);
  c.Mb_ros = c.Mbochat / c.ros;
  c.r_Tod = 1.0 / c.Tod;
  c.r_Ufr2 = 1.0 / (c.Ufr * c.Ufr);
  c.Dxr_m03 = std::pow(c.Dxr, -0.3);
  c.qb_k = 0.053 * std::sqrt((c.Sx - 1) * c.g) * std::pow(c.dm, 1.5);
}

}  // namespace

struct HydistHandle {
  int device = 0;
  cudaStream_t stream = nullptr;
  // S holds the FP64 form's state; in the FP32 form Sf holds it and S only
  // the fields common to both (dimensions, water level, bed, mask, tables,
  // series, clock), so that form-independent code reads S alone
  State S{};
  Coef c{};
  bool fp32 = false;
  StateT<float> Sf{};
  CoefT<float> cf{};
  HydistOptions o{};
  double t = 0;
  std::vector<void*> allocs;
  // device memory: the allocation sequence runs once with `planning` set,
  // recording the arrays' sizes, then again carving them out of chunks of
  // up to CHUNK bytes, one for a scenario of up to a few thousand cells a
  // side (each cudaMalloc call costs about 0.4 ms, whatever its size: 45
  // separate ones made hydist_create of a 2048x1024 scenario take 100 ms
  // against 9 ms)
  static constexpr size_t CHUNK = (size_t)4 << 30;
  bool planning = false;
  std::vector<size_t> plan;
  size_t plan_idx = 0;
  char* chunk = nullptr;
  size_t chunk_size = 0, chunk_used = 0;
  double* mass_part = nullptr;  // per-block partial sums
  unsigned* mass_done = nullptr;  // blocks finished, reset by the last one
  double* mass_host = nullptr;    // the result, in mapped pinned host memory
  double* mass_host_dev = nullptr;
  int mass_blocks = 0;
  // one captured step per sediment phase: [bed*4 + sed_x*2 + sed_y]
  cudaGraphExec_t graph[8] = {};
  long long graph_launches[8] = {};
  Trace trace;                                    // kernel launch counter
  cudaEvent_t ev[PH_COUNT + 1] = {};
  cudaEvent_t kev[2 * KS_COUNT] = {};
  int next_half = 0;  // 1 while the second half of a step is pending
  // host time of hydist_create by part (ms): device allocation and zeroing,
  // input copies, set-up kernels, total
  double create_ms[4] = {};
};

namespace {

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// One memory pool per device for the handles' arrays, keeping what destroyed
// handles release (release threshold unlimited): a create after a destroy
// reuses device pages that are already mapped instead of asking the driver
// for new ones, which on a GPU's first use of the memory costs tens of ms
// per GB. The pool's memory goes back to the driver at process exit.
cudaMemPool_t handle_pool(int dev) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

// The launchers of the handle's form: f(state, coefficients).
template <class F>
void on_state(HydistHandle* h, F&& f) {
  if (h->fp32) f(h->Sf, h->cf);
  else f(h->S, h->c);
}

// granule and footprint of an array of `raw` bytes: arrays of 2 MiB or more
// start on, and fill, whole 2 MiB granules as separate cudaMalloc calls
// place them; smaller ones take 256-byte steps
inline void granule(size_t raw, size_t& g, size_t& bytes) {
  g = raw >= ((size_t)2 << 20) ? ((size_t)2 << 20) : 256;
  bytes = (raw + g - 1) / g * g;
}

// a zeroed device array of n values, carved out of the handle's chunks in
// the order the sizing pass recorded (a request beyond that record gets a
// cudaMalloc of its own)
template <class T>
int dalloc(HydistHandle* h, T** p, size_t n) {
  const size_t raw = n * sizeof(T) + 64;
  if (h->planning) {
    // sizing pass: a placeholder that is never dereferenced
    h->plan.push_back(raw);
    *p = reinterpret_cast<T*>((uintptr_t)256);
    return HYDIST_OK;
  }
  size_t g, bytes;
  granule(raw, g, bytes);
  if (h->plan_idx < h->plan.size()) {
    size_t off = (h->chunk_used + g - 1) / g * g;
    if (!h->chunk || off + bytes > h->chunk_size) {
      // a new chunk for this and the next recorded arrays, up to CHUNK
      size_t sz = 0;
      for (size_t j = h->plan_idx; j < h->plan.size(); ++j) {
        size_t gj, bj;
        granule(j == h->plan_idx ? raw : h->plan[j], gj, bj);
        const size_t o = (sz + gj - 1) / gj * gj;
        if (j > h->plan_idx && o + bj > HydistHandle::CHUNK) break;
        sz = o + bj;
      }
      void* q = nullptr;
      const auto ta = Clock::now();
      cudaMemPool_t pool = handle_pool(h->device);
      if (!pool) return fail(HYDIST_ERR_CUDA, "no device memory pool");
      CK(cudaMallocFromPoolAsync(&q, sz, pool, h->stream));
      h->allocs.push_back(q);
      CK(cudaMemsetAsync(q, 0, sz, h->stream));
      CK(cudaStreamSynchronize(h->stream));
      h->create_ms[0] += ms_since(ta);
      h->chunk = static_cast<char*>(q);
      h->chunk_size = sz;
      off = 0;
    }
    *p = reinterpret_cast<T*>(h->chunk + off);
    h->chunk_used = off + bytes;
    ++h->plan_idx;
    return HYDIST_OK;
  }
  void* q = nullptr;
  cudaMemPool_t pool = handle_pool(h->device);
  if (!pool) return fail(HYDIST_ERR_CUDA, "no device memory pool");
  CK(cudaMallocFromPoolAsync(&q, raw, pool, h->stream));
  CK(cudaMemsetAsync(q, 0, raw, h->stream));
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return HYDIST_OK;
}

#define TRY(x)                    \
  do {                            \
    int r__ = (x);                \
    if (r__ != HYDIST_OK) return r__; \
  } while (0)

int check_device_err(HydistHandle* h) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, h->S.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (e & DEV_SEG_OVERFLOW) return fail(HYDIST_ERR_SEGMENTS, "a line has more than 20 wet segments");
  if (e & DEV_NONFINITE)
    return fail(HYDIST_ERR_NONFINITE, "a NaN or Inf was committed to u, v, z or the concentration");
  return HYDIST_OK;
}

// The boundary update interpolates hour floor(t/3600) and the next one
// (support_funcs.cpp:624); refuse steps whose time runs past the series.
int check_horizon(HydistHandle* h, int nsteps) {
  const double t_end = h->t + nsteps * h->c.dT;
  if ((int)((double)(float)t_end / 3600) + 1 > h->S.T - 1)
    return fail(HYDIST_ERR_ARG, "boundary series too short for the requested steps");
  return HYDIST_OK;
}

// one full step (engine.cpp:65-295); the sediment gates (engine.cpp:149,
// 258) are decided on the host, the time itself advances on the device
void enqueue_step(HydistHandle* h, bool sed_x, bool sed_y, bool bed, Trace* tr) {
  on_state(h, [&](auto& St, auto& Cf) {
    launch_half_x(St, Cf, sed_x, h->stream, tr);
    if (sed_x) launch_sediment(St, Cf, true, false, h->stream, tr);
    else if (tr && tr->ev) cudaEventRecord(tr->ev[PH_SEDIMENT_X + 1], h->stream);
    launch_half_y(St, Cf, sed_y, h->stream, tr, {}, sed_y && bed);
    if (sed_y) launch_sediment(St, Cf, false, bed, h->stream, tr);
    else if (tr && tr->ev) cudaEventRecord(tr->ev[PH_SEDIMENT_Y + 1], h->stream);
  });
}

// the bed change runs after the j-sweep of a step ending at t2 once both the
// sweeps and the bed change have started
bool bed_on(const HydistHandle* h, double t2) {
  return h->o.bed_change && t2 >= h->o.sediment_start && t2 >= h->o.bed_change_start;
}

int set_device_clock(HydistHandle* h) {
  if (h->planning) return HYDIST_OK;
  CK(cudaMemcpyAsync(h->S.clock, &h->t, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return HYDIST_OK;
}

// Volume of the wet cells, sum of (htaiz + z) over rows 2..N and columns
// 2..M where khouot == 0, FP64. Each block sums whole rows into part[]; the
// last block to finish adds the partial sums in block order (the same
// result every call) and writes it to mapped host memory.
__global__ void k_mass(State S, double* part, unsigned* done, double* out) {
  __shared__ double sh[256];
  __shared__ bool last;
  double acc = 0;
  for (int i = blockIdx.x + 2; i <= S.N; i += gridDim.x) {
    const int row = i * S.W;
    for (int j = threadIdx.x + 2; j <= S.M; j += blockDim.x)
      if (S.khouot[row + j] == 0) acc += S.htaiz[row + j] + S.z[row + j];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = sh[0];
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  acc = 0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) acc += part[k];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *out = sh[0];
    __threadfence_system();
    *done = 0;
  }
}

// A field's device array and element size (8, or 4 for the FP32 form's
// single-precision fields).
struct FieldRef {
  void* p = nullptr;
  int esz = 8;
};

template <class R>
FieldRef bulk_field(const StateT<R>& S, int f) {
  auto r = [](const R* q) { return FieldRef{const_cast<R*>(q), (int)sizeof(R)}; };
  switch (f) {
    case HYDIST_FIELD_U: return r(S.u);
    case HYDIST_FIELD_V: return r(S.v);
    case HYDIST_FIELD_FS: return r(S.FS);
    case HYDIST_FIELD_TFS: return r(S.tFS);
    case HYDIST_FIELD_H_MOI: return r(S.Hmoi);
    case HYDIST_FIELD_HTDU: return r(S.Htdu);
    case HYDIST_FIELD_HTDV: return r(S.Htdv);
    case HYDIST_FIELD_TU: return r(S.tu);
    case HYDIST_FIELD_TV: return r(S.tv);
    case HYDIST_FIELD_KX1: return r(S.Kx1);
    case HYDIST_FIELD_KY1: return r(S.Ky1);
    case HYDIST_FIELD_VTH: return r(S.VTH);
    case HYDIST_FIELD_KX: return r(S.Kx);
    case HYDIST_FIELD_KY: return r(S.Ky);
    case HYDIST_FIELD_QBX: return r(S.Qbx);
    case HYDIST_FIELD_QBY: return r(S.Qby);
    default: return FieldRef{};
  }
}

FieldRef field_ref(HydistHandle* h, int f) {
  const State& S = h->S;
  switch (f) {
    case HYDIST_FIELD_Z: return FieldRef{S.z, 8};
    case HYDIST_FIELD_TZ: return FieldRef{S.tz, 8};
    case HYDIST_FIELD_DH: return FieldRef{S.dH, 8};
    case HYDIST_FIELD_H: return FieldRef{const_cast<double*>(S.h), 8};
    case HYDIST_FIELD_HTAIZ: return FieldRef{const_cast<double*>(S.htaiz), 8};
    default: return h->fp32 ? bulk_field(h->Sf, f) : bulk_field(h->S, f);
  }
}

// n values of a field to host FP64 / from host FP64 (synchronous)
int field_to_host(HydistHandle* h, const FieldRef& r, double* host, size_t n) {
  if (r.esz == 8) {
    CK(cudaMemcpyAsync(host, r.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return HYDIST_OK;
  }
  std::vector<float> tmp(n);
  CK(cudaMemcpyAsync(tmp.data(), r.p, n * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (size_t k = 0; k < n; ++k) host[k] = tmp[k];
  return HYDIST_OK;
}

int field_from_host(HydistHandle* h, const FieldRef& r, const double* host, size_t n) {
  if (r.esz == 8) {
    CK(cudaMemcpyAsync(r.p, host, n * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return HYDIST_OK;
  }
  std::vector<float> tmp(host, host + n);
  CK(cudaMemcpyAsync(r.p, tmp.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return HYDIST_OK;
}

}  // namespace

namespace hyd {
// Lets the other translation units of the library set the message that
// hydist_last_error() returns.
void set_last_error(const char* m) { g_err = m; }
}  // namespace hyd

extern "C" {

const char* hydist_last_error(void) { return g_err.c_str(); }
const char* hydist_version(void) { return "hydist_b200 0.1 (sm_100a)"; }

void hydist_params_default(HydistParams* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->dX = 10.0;
  p->dY = 10.0;
  p->dT = 2;
  p->NANGDAY = 0.0;
  p->H_TINH = 0.02;
  p->heso = 0.94;
  p->mu_mn = 0.2;
  p->NDnen = 0.00;
  p->Tod = 0.06;
  p->Toe = 0.15;
  p->hstoe = 0;
  p->ghtoe = 3;
  p->Mbochat = 0.00001;
  p->ro = 1000;
  p->ros = 2000;
  p->dm = 0.00001;
  p->d90 = 0.002;
  p->muy = 1.01e-06;
  p->Dorong = 0.5;
  p->Sx = 2;
  p->CORIOLIS_FORCE = 0.0;
  p->g = 9.81;
  p->Wind = 0.0;
  p->huonggio = 0.0;
  p->wss = -1;
  p->Ks = -1;
}

void hydist_options_default(HydistOptions* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->t_start = 0;
  o->sediment_start = 20 * 3600;
  o->bed_change_start = 500 * 3600;
  o->ketdinh = 1;
  o->bed_change = 0;
  o->precision = HYDIST_FP64;
}

void hydist_bienq_from_boundary_type(const int32_t* bt, int32_t n, int32_t bienQ[4]) {
  for (int k = 0; k < 4; ++k) bienQ[k] = (bt && k < n && bt[k] == 2) ? 1 : 0;
}

}  // extern "C"

namespace {

int check_params(const HydistParams* p, const HydistOptions* o) {
  if (!(p->dX > 0 && p->dY > 0 && p->dT > 0)) return fail(HYDIST_ERR_ARG, "dX, dY, dT must be > 0");
  if (o->precision != HYDIST_FP64 && o->precision != HYDIST_FP32_REFINE &&
      o->precision != HYDIST_FP32)
    return fail(HYDIST_ERR_ARG, "unknown precision");
  for (int32_t f : {o->ketdinh, o->bed_change, o->kenhhepd, o->kenhhepng, o->channel_wave,
                    o->reset_horizontal, o->bed_feedback})
    if (f != 0 && f != 1) return fail(HYDIST_ERR_ARG, "option flags must be 0 or 1");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(HYDIST_ERR_NODEVICE, "no CUDA device");
  return HYDIST_OK;
}

// Handle, stream and constants of a new scenario (no arrays yet).
int new_handle(const HydistParams* p, const HydistOptions* o, int device, int M, int N, int T,
               const int32_t bienQ[4], HydistHandle** out) {
  auto* h = new HydistHandle();
  *out = h;
  if (device < 0) cudaGetDevice(&device);
  h->device = device;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  derive(*p, h->c);
  h->fp32 = o->precision == HYDIST_FP32_REFINE || o->precision == HYDIST_FP32;
  h->cf = CoefT<float>::from(h->c);
  h->o = *o;
  h->t = o->t_start;
  State& S = h->S;
  S.M = M;
  S.N = N;
  S.W = S.M + 3;
  S.H = S.N + 3;
  S.T = T;
  for (int k = 0; k < 4; ++k) S.bienQ[k] = bienQ[k] ? 1 : 0;
  S.ketdinh = o->ketdinh ? 1 : 0;
  S.race_new = 1;
  S.refine = o->precision == HYDIST_FP32_REFINE ? 1 : 0;
  // the reference's channel = kenhhepd xor kenhhepng (engine.h:33)
  const bool channel = (o->kenhhepd != 0) != (o->kenhhepng != 0);
  S.chan = channel ? (o->channel_wave ? 2 : 1) : 0;
  S.x_lo = channel && o->kenhhepd ? 3 : 2;
  S.x_hi = channel && o->kenhhepd ? M - 1 : M;
  S.y_lo = channel && o->kenhhepng ? 3 : 2;
  S.reset_h = o->reset_horizontal ? 1 : 0;
  S.bed_fb = o->bed_change && o->bed_feedback ? 1 : 0;
  S.src_start = o->bed_change_start;
  return HYDIST_OK;
}

// The arrays only this library uses: smoothing buffers, boundary weights,
// line-solver scratch, flags, counters, the device clock.
// The FP64 / FP32 arrays only this library uses: smoothing buffers and the
// line-solver scratch (3 values per unknown, 4 lines per slot, one slot per
// CTA of the persistent sweep grid).
template <class R>
int bulk_private(HydistHandle* h, StateT<R>& B) {
  const State& S = h->S;
  const size_t n = (size_t)S.W * S.H;
  TRY(dalloc(h, &B.tmp, n));
  TRY(dalloc(h, &B.sv, n));
  TRY(dalloc(h, &B.pre, 4 * n));
  B.su = B.tmp;
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
  B.lslots = 2 * nsm;
  const size_t U = (size_t)2 * std::max(S.M, S.N);
  // at least 4 (max(M,N)+3) doubles: preprocess_data borrows it as FP64;
  // the refined FP32 form keeps 7 values per unknown (its refinement stores
  // the rows)
  const size_t arrays = S.refine ? 7 : 3;
  TRY(dalloc(h, &B.lscratch, std::max((size_t)B.lslots * arrays * U * 4, 8 * U + 64)));
  return HYDIST_OK;
}

// The arrays only this library uses: the above, the boundary weights,
// flags, counters, the device clock.
int private_arrays(HydistHandle* h) {
  State& S = h->S;
  TRY(dalloc(h, &S.hi, 2 * (S.M + S.N + 6)));
  TRY(dalloc(h, &S.hmax, 4));
  TRY(dalloc(h, &S.err, 4));
  TRY(dalloc(h, &S.colflag, S.W));
  TRY(dalloc(h, &S.rowflag, S.H));
  TRY(dalloc(h, &S.segcnt, 2 * S.H + 2 * S.W));
  TRY(dalloc(h, &S.clock, 4));
  TRY(set_device_clock(h));
  h->mass_blocks = 296;
  TRY(dalloc(h, &h->mass_part, h->mass_blocks + 1));
  TRY(dalloc(h, &h->mass_done, 1));
  if (!h->planning && !h->mass_host) {
    CK(cudaHostAlloc((void**)&h->mass_host, sizeof(double), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void**)&h->mass_host_dev, h->mass_host, 0));
  }
  return h->fp32 ? bulk_private(h, h->Sf) : bulk_private(h, h->S);
}

// a device array of n values of type R from host FP64 (converted; synchronous)
template <class R>
int upload_new(HydistHandle* h, R** dst, const double* host, size_t n) {
  TRY(dalloc(h, dst, n));
  if (!host || h->planning) return HYDIST_OK;
  const auto t0 = Clock::now();
  struct Acc {
    double& ms;
    Clock::time_point t0;
    ~Acc() { ms += ms_since(t0); }
  } acc{h->create_ms[1], t0};
  if (sizeof(R) == 8) {
    CK(cudaMemcpyAsync(*dst, host, n * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<R> tmp(host, host + n);
    CK(cudaMemcpyAsync(*dst, tmp.data(), n * sizeof(R), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  return HYDIST_OK;
}

// the fields of the step's type R: static inputs (ν, Fw), derived statics
// (Kx1, Ky1, Tsxw, Tsyw), the velocity/depth/concentration state and the
// boundary velocities
template <class R>
int bulk_arrays(HydistHandle* h, StateT<R>& B, const HydistScenario* sc) {
  const State& S = h->S;
  const size_t n = (size_t)S.W * S.H;
  R* tmp;
  TRY(upload_new(h, &tmp, sc->visco, n));
  B.visco = tmp;
  TRY(upload_new(h, &tmp, sc->Fw, n));
  B.Fw = tmp;
  const R** st_static[] = {&B.Kx1, &B.Ky1, &B.Tsxw, &B.Tsyw};
  for (const R** q : st_static) {
    TRY(dalloc(h, &tmp, n));
    *q = tmp;
  }
  R** st[] = {&B.u, &B.v, &B.tu, &B.tv, &B.Hmoi, &B.Htdu, &B.Htdv, &B.VTH, &B.Kx, &B.Ky, &B.Qbx,
              &B.Qby};
  for (R** q : st) TRY(dalloc(h, q, n));
  TRY(upload_new(h, &B.FS, sc->FS0, n));
  TRY(upload_new(h, &B.tFS, sc->FS0, n));
  TRY(dalloc(h, &B.ubt, S.W));
  TRY(dalloc(h, &B.ubp, S.W));
  TRY(dalloc(h, &B.vbt, S.H));
  TRY(dalloc(h, &B.vbd, S.H));
  return HYDIST_OK;
}

// the fields common to both forms, from S into the FP32 form's state
void mirror_common(HydistHandle* h) {
  const State& S = h->S;
  StateT<float>& F = h->Sf;
  F.M = S.M;
  F.N = S.N;
  F.W = S.W;
  F.H = S.H;
  F.T = S.T;
  for (int k = 0; k < 4; ++k) F.bienQ[k] = S.bienQ[k];
  F.ketdinh = S.ketdinh;
  F.race_new = S.race_new;
  F.refine = S.refine;
  F.chan = S.chan;
  F.x_lo = S.x_lo;
  F.x_hi = S.x_hi;
  F.y_lo = S.y_lo;
  F.reset_h = S.reset_h;
  F.bed_fb = S.bed_fb;
  F.src_start = S.src_start;
  F.h0 = S.h0;
  F.htaiz0 = S.htaiz0;
  F.h = S.h;
  F.hsnham = S.hsnham;
  F.htaiz = S.htaiz;
  F.htaiz_bd = S.htaiz_bd;
  F.z = S.z;
  F.tz = S.tz;
  F.dH = S.dH;
  F.khouot = S.khouot;
  F.hi = S.hi;
  F.hmax = S.hmax;
  for (int k = 0; k < 4; ++k) {
    F.bc[k] = S.bc[k];
    F.CC[k] = S.CC[k];
  }
  F.btype = S.btype;
  F.daui = S.daui;
  F.cuoii = S.cuoii;
  F.moci = S.moci;
  F.dauj = S.dauj;
  F.cuoij = S.cuoij;
  F.mocj = S.mocj;
  F.err = S.err;
  F.colflag = S.colflag;
  F.rowflag = S.rowflag;
  F.segcnt = S.segcnt;
  F.clock = S.clock;
}

// Runs the allocation sequence `f` once to record its arrays' sizes, then
// again with the arrays carved out of a few zeroed chunks.
template <class F>
int with_arena(HydistHandle* h, F&& f) {
  h->planning = true;
  h->plan.clear();
  const int rc = f();
  h->planning = false;
  if (rc != HYDIST_OK) return rc;
  h->plan_idx = 0;
  h->chunk = nullptr;
  h->chunk_size = h->chunk_used = 0;
  return f();
}

}  // namespace

extern "C" {

int hydist_create(const HydistScenario* sc, const HydistParams* p, const HydistOptions* o,
                  int device, HydistHandle** out) {
  if (!sc || !p || !o || !out) return fail(HYDIST_ERR_ARG, "null argument");
  *out = nullptr;
  if (sc->M < 4 || sc->N < 4 || sc->total_time < 2)
    return fail(HYDIST_ERR_ARG, "mesh must be at least 4x4 and series at least 2 hours long");
  if (!sc->h || !sc->hsnham || !sc->visco || !sc->Fw || !sc->boundary_type)
    return fail(HYDIST_ERR_ARG, "missing input array");
  if (sc->n_boundary_type < 4 * SEG)
    return fail(HYDIST_ERR_ARG, "boundary_type needs 4 sides x 20 segments");
  TRY(check_params(p, o));
  const auto t_create = Clock::now();
  HydistHandle* h = nullptr;
  int rc = new_handle(p, o, device, sc->M, sc->N, sc->total_time, sc->bienQ, &h);
  if (rc == HYDIST_OK) rc = with_arena(h, [&]() -> int {
    State& S = h->S;
    const size_t n = (size_t)S.W * S.H;
    double* tmp;
    // FP64 in both forms: bed, water level, bed change, series
    TRY(upload_new(h, &tmp, sc->h, n));
    S.h = tmp;
    TRY(upload_new(h, &tmp, sc->hsnham, n));
    S.hsnham = tmp;
    const double* bcs[4] = {sc->bc_up, sc->bc_down, sc->bc_left, sc->bc_right};
    const double* ccs[4] = {sc->CC_up, sc->CC_down, sc->CC_left, sc->CC_right};
    for (int k = 0; k < 4; ++k) {
      TRY(upload_new(h, &tmp, bcs[k], S.T));
      S.bc[k] = tmp;
      TRY(upload_new(h, &tmp, ccs[k], S.T));
      S.CC[k] = tmp;
    }
    int* itmp;
    TRY(dalloc(h, &itmp, 4 * SEG));
    if (!h->planning)
      CK(cudaMemcpyAsync(itmp, sc->boundary_type, 4 * SEG * 4, cudaMemcpyHostToDevice, h->stream));
    S.btype = itmp;
    TRY(dalloc(h, &tmp, n));
    S.htaiz = tmp;
    TRY(dalloc(h, &tmp, n));
    S.htaiz_bd = tmp;
    if (S.bed_fb) {
      // the initial bed, copied after the set-up kernels
      TRY(dalloc(h, &tmp, n));
      S.h0 = tmp;
      TRY(dalloc(h, &tmp, n));
      S.htaiz0 = tmp;
    }
    TRY(upload_new(h, &S.z, sc->z0, n));
    TRY(upload_new(h, &S.tz, sc->z0, n));
    TRY(dalloc(h, &S.dH, n));
    TRY(dalloc(h, &S.khouot, n));
    TRY(dalloc(h, &S.daui, S.H * SEG));
    TRY(dalloc(h, &S.cuoii, S.H * SEG));
    TRY(dalloc(h, &S.moci, S.H));
    TRY(dalloc(h, &S.dauj, S.W * SEG));
    TRY(dalloc(h, &S.cuoij, S.W * SEG));
    TRY(dalloc(h, &S.mocj, S.W));
    // the step's type: FP64, or FP32 in the FP32 form
    if (h->fp32) TRY(bulk_arrays(h, h->Sf, sc));
    else TRY(bulk_arrays(h, h->S, sc));
    TRY(private_arrays(h));
    if (h->fp32) mirror_common(h);
    return HYDIST_OK;
  });
  if (rc == HYDIST_OK) rc = [&]() -> int {
    const auto t_init = Clock::now();
    on_state(h, [&](auto& St, auto& Cf) { launch_init(St, Cf, h->stream); });
    CK(cudaGetLastError());
    const size_t nb = (size_t)h->S.W * h->S.H * sizeof(double);
    if (h->S.bed_fb) {
      CK(cudaMemcpyAsync(const_cast<double*>(h->S.h0), h->S.h, nb, cudaMemcpyDeviceToDevice,
                         h->stream));
      CK(cudaMemcpyAsync(const_cast<double*>(h->S.htaiz0), h->S.htaiz, nb,
                         cudaMemcpyDeviceToDevice, h->stream));
    }
    TRY(check_device_err(h));
    h->create_ms[2] = ms_since(t_init);
    return HYDIST_OK;
  }();
  if (rc != HYDIST_OK) {
    hydist_destroy(h);
    return rc;
  }
  h->create_ms[3] = ms_since(t_create);
  *out = h;
  return HYDIST_OK;
}

int hydist_create_phases(const HydistHandle* h, double* ms) {
  if (!h || !ms) return fail(HYDIST_ERR_ARG, "null argument");
  for (int k = 0; k < 4; ++k) ms[k] = h->create_ms[k];
  return HYDIST_OK;
}

int hydist_create_external(const HydistExternal* e, const HydistParams* p, const HydistOptions* o,
                           int device, HydistHandle** out) {
  if (!e || !p || !o || !out) return fail(HYDIST_ERR_ARG, "null argument");
  *out = nullptr;
  if (e->M < 4 || e->N < 4 || e->total_time < 2)
    return fail(HYDIST_ERR_ARG, "mesh must be at least 4x4 and series at least 2 hours long");
  const void* need[] = {e->h, e->hsnham, e->visco, e->Fw, e->htaiz, e->htaiz_bd, e->Kx1, e->Ky1,
                        e->Tsxw, e->Tsyw, e->bc_up, e->bc_down, e->bc_left, e->bc_right,
                        e->CC_up, e->CC_down, e->CC_left, e->CC_right, e->boundary_type,
                        e->u, e->v, e->z, e->t_u, e->t_v, e->t_z, e->H_moi, e->Htdu, e->Htdv,
                        e->FS, e->tFS, e->VTH, e->Kx, e->Ky, e->dH, e->Qbx, e->Qby, e->khouot,
                        e->daui, e->cuoii, e->moci, e->dauj, e->cuoij, e->mocj, e->ubt, e->ubp,
                        e->vbt, e->vbd};
  for (const void* q : need)
    if (!q) return fail(HYDIST_ERR_ARG, "missing device array");
  TRY(check_params(p, o));
  if (o->precision != HYDIST_FP64)
    return fail(HYDIST_ERR_ARG, "caller-owned arrays are FP64: use HYDIST_FP64");
  if (o->bed_change && o->bed_feedback)
    return fail(HYDIST_ERR_ARG,
                "bed_feedback rewrites h, htaiz, Kx1 and Ky1, which an external handle only reads");
  HydistHandle* h = nullptr;
  int rc = new_handle(p, o, device, e->M, e->N, e->total_time, e->bienQ, &h);
  if (rc == HYDIST_OK) rc = [&]() -> int {
    State& S = h->S;
    S.h = e->h;
    S.hsnham = e->hsnham;
    S.visco = e->visco;
    S.Fw = e->Fw;
    S.htaiz = e->htaiz;
    S.htaiz_bd = e->htaiz_bd;
    S.Kx1 = e->Kx1;
    S.Ky1 = e->Ky1;
    S.Tsxw = e->Tsxw;
    S.Tsyw = e->Tsyw;
    S.bc[0] = e->bc_up;
    S.bc[1] = e->bc_down;
    S.bc[2] = e->bc_left;
    S.bc[3] = e->bc_right;
    S.CC[0] = e->CC_up;
    S.CC[1] = e->CC_down;
    S.CC[2] = e->CC_left;
    S.CC[3] = e->CC_right;
    S.btype = e->boundary_type;
    S.u = e->u;
    S.v = e->v;
    S.z = e->z;
    S.tu = e->t_u;
    S.tv = e->t_v;
    S.tz = e->t_z;
    S.Hmoi = e->H_moi;
    S.Htdu = e->Htdu;
    S.Htdv = e->Htdv;
    S.FS = e->FS;
    S.tFS = e->tFS;
    S.VTH = e->VTH;
    S.Kx = e->Kx;
    S.Ky = e->Ky;
    S.dH = e->dH;
    S.Qbx = e->Qbx;
    S.Qby = e->Qby;
    S.khouot = e->khouot;
    S.daui = e->daui;
    S.cuoii = e->cuoii;
    S.moci = e->moci;
    S.dauj = e->dauj;
    S.cuoij = e->cuoij;
    S.mocj = e->mocj;
    S.ubt = e->ubt;
    S.ubp = e->ubp;
    S.vbt = e->vbt;
    S.vbd = e->vbd;
    TRY(with_arena(h, [&]() { return private_arrays(h); }));
    // the boundary discharge weights from the caller's depths; everything
    // else was set up by the caller (Onetime_init, the segment scans and
    // Htuongdoi, as the reference's main does before the time loop)
    launch_preprocess(S, h->c, h->stream);
    CK(cudaGetLastError());
    TRY(check_device_err(h));
    return HYDIST_OK;
  }();
  if (rc != HYDIST_OK) {
    hydist_destroy(h);
    return rc;
  }
  *out = h;
  return HYDIST_OK;
}

int hydist_half_step(HydistHandle* h, int32_t half) {
  if (!h) return fail(HYDIST_ERR_ARG, "null handle");
  if (half != 0 && half != 1) return fail(HYDIST_ERR_ARG, "half must be 0 or 1");
  if (half != h->next_half)
    return fail(HYDIST_ERR_STATE, half == 0 ? "the second half-step is pending"
                                            : "the first half-step has not run");
  CK(cudaSetDevice(h->device));
  if (half == 0) TRY(check_horizon(h, 1));
  const double t = h->t + 0.5 * h->c.dT;
  const bool sed = t >= h->o.sediment_start;
  if (half == 0) {
    on_state(h, [&](auto& St, auto& Cf) {
      launch_half_x(St, Cf, sed, h->stream, &h->trace);
      if (sed) launch_sediment(St, Cf, true, false, h->stream, &h->trace);
    });
  } else {
    on_state(h, [&](auto& St, auto& Cf) {
      const bool bed = sed && bed_on(h, t);
      launch_half_y(St, Cf, sed, h->stream, &h->trace, {}, bed);
      if (sed) launch_sediment(St, Cf, false, bed, h->stream, &h->trace);
    });
  }
  h->t = t;
  h->next_half = 1 - half;
  CK(cudaGetLastError());
  return HYDIST_OK;
}

int hydist_update_boundary(HydistHandle* h, double t) {
  if (!h) return fail(HYDIST_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  const double keep = h->t;
  h->t = t;
  int rc = set_device_clock(h);
  if (rc == HYDIST_OK) {
    on_state(h, [&](auto& St, auto& Cf) { launch_boundary(St, Cf, h->stream); });
    h->trace.launches += 1;
    rc = cudaGetLastError() == cudaSuccess ? HYDIST_OK : fail(HYDIST_ERR_CUDA, "boundary launch failed");
  }
  h->t = keep;
  const int rc2 = set_device_clock(h);
  return rc != HYDIST_OK ? rc : rc2;
}

int hydist_destroy(HydistHandle* h) {
  if (!h) return HYDIST_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto& g : h->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  // back into the device's pool (see handle_pool)
  for (void* p : h->allocs) cudaFreeAsync(p, h->stream);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->mass_host) cudaFreeHost(h->mass_host);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return HYDIST_OK;
}

int hydist_step(HydistHandle* h, int32_t nsteps) {
  if (!h) return fail(HYDIST_ERR_ARG, "null handle");
  if (h->next_half) return fail(HYDIST_ERR_STATE, "the second half-step is pending");
  if (nsteps < 0) return fail(HYDIST_ERR_ARG, "negative step count");
  CK(cudaSetDevice(h->device));
  TRY(check_horizon(h, nsteps));
  for (int k = 0; k < nsteps; ++k) {
    const double t1 = h->t + 0.5 * h->c.dT;
    const double t2 = t1 + h->c.dT * 0.5;
    enqueue_step(h, t1 >= h->o.sediment_start, t2 >= h->o.sediment_start, bed_on(h, t2),
                 &h->trace);
    h->t = t2;
  }
  CK(cudaGetLastError());
  return HYDIST_OK;
}

int hydist_step_traced_sweeps(HydistHandle* h, float* phase_ms, float* sweep_ms) {
  if (!h || !phase_ms) return fail(HYDIST_ERR_ARG, "null argument");
  if (h->next_half) return fail(HYDIST_ERR_STATE, "the second half-step is pending");
  CK(cudaSetDevice(h->device));
  TRY(check_horizon(h, 1));
  if (!h->ev[0])
    for (auto& e : h->ev) CK(cudaEventCreate(&e));
  if (sweep_ms && !h->kev[0])
    for (auto& e : h->kev) CK(cudaEventCreate(&e));
  Trace tr;
  tr.ev = h->ev;
  if (sweep_ms) tr.kev = h->kev;
  const double t1 = h->t + 0.5 * h->c.dT;
  const double t2 = t1 + h->c.dT * 0.5;
  CK(cudaEventRecord(h->ev[0], h->stream));
  enqueue_step(h, t1 >= h->o.sediment_start, t2 >= h->o.sediment_start, bed_on(h, t2), &tr);
  h->trace.launches += tr.launches;
  h->t = t2;
  CK(cudaGetLastError());
  CK(cudaEventSynchronize(h->ev[PH_COUNT]));
  for (int p = 0; p < PH_COUNT; ++p) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->ev[p], h->ev[p + 1]));
    phase_ms[p] = ms;
  }
  if (sweep_ms) {
    for (int k = 0; k < KS_COUNT; ++k) {
      float ms = 0;
      if (tr.krec[k]) CK(cudaEventElapsedTime(&ms, h->kev[2 * k], h->kev[2 * k + 1]));
      sweep_ms[k] = ms;
    }
  }
  return HYDIST_OK;
}

int hydist_step_traced(HydistHandle* h, float* phase_ms) {
  return hydist_step_traced_sweeps(h, phase_ms, nullptr);
}

int hydist_kernel_launches(HydistHandle* h, int64_t* count) {
  if (!h || !count) return fail(HYDIST_ERR_ARG, "null argument");
  *count = h->trace.launches;
  return HYDIST_OK;
}

int hydist_step_graph(HydistHandle* h, int32_t nsteps) {
  // The time advances on the device, so the launches of a step are the same
  // every step: one graph per sediment phase, captured on first use.
  if (!h) return fail(HYDIST_ERR_ARG, "null handle");
  if (h->next_half) return fail(HYDIST_ERR_STATE, "the second half-step is pending");
  if (nsteps < 0) return fail(HYDIST_ERR_ARG, "negative step count");
  CK(cudaSetDevice(h->device));
  TRY(check_horizon(h, nsteps));
  for (int k = 0; k < nsteps; ++k) {
    const double t1 = h->t + 0.5 * h->c.dT;
    const double t2 = t1 + h->c.dT * 0.5;
    const bool sx = t1 >= h->o.sediment_start, sy = t2 >= h->o.sediment_start;
    const bool bd = bed_on(h, t2);
    const int gi = (bd ? 4 : 0) + (sx ? 2 : 0) + (sy ? 1 : 0);
    cudaGraphExec_t& ex = h->graph[gi];
    if (!ex) {
      cudaGraph_t g = nullptr;
      Trace tr;
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      enqueue_step(h, sx, sy, bd, &tr);
      CK(cudaStreamEndCapture(h->stream, &g));
      h->graph_launches[gi] = tr.launches;
      const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      CK(e);
    }
    CK(cudaGraphLaunch(ex, h->stream));
    h->trace.launches += h->graph_launches[gi];
    h->t = t2;
  }
  return HYDIST_OK;
}

int hydist_sync(HydistHandle* h) {
  if (!h) return fail(HYDIST_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  return check_device_err(h);
}

int hydist_get_time(HydistHandle* h, double* t) {
  if (!h || !t) return fail(HYDIST_ERR_ARG, "null argument");
  *t = h->t;
  return HYDIST_OK;
}

// ---- ensembles: many scenarios stepped by one graph launch -------------
struct HydistEnsemble {
  int device = 0;
  std::vector<HydistHandle*> m;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join;
  // one graph per pattern of the members' sediment phases
  std::map<std::vector<unsigned char>, std::pair<cudaGraphExec_t, long long>> graphs;
  // batched stepping: members of one mesh size and form, whose states and
  // coefficients are copied to the device once, so that each kernel of a
  // step is one launch over all members (uniform: they allow it; batched:
  // it is used when the members' sediment phases agree)
  bool uniform = false, batched = false;
  void *bS = nullptr, *bC = nullptr;  // StateT<R>[n], CoefT<R>[n]
};

}  // extern "C"

namespace {

// members that can share launches: same mesh, form and launch-shaping
// options
bool same_launches(const HydistHandle* a, const HydistHandle* b) {
  return a->S.M == b->S.M && a->S.N == b->S.N && a->fp32 == b->fp32 && a->S.refine == b->S.refine &&
         a->S.x_lo == b->S.x_lo && a->S.x_hi == b->S.x_hi && a->S.y_lo == b->S.y_lo &&
         a->S.reset_h == b->S.reset_h && a->S.bed_fb == b->S.bed_fb &&
         a->S.lslots == b->S.lslots && a->Sf.lslots == b->Sf.lslots;
}

// one step of every member of a batch, on stream st
template <class R>
void enqueue_step_batch(const StateT<R>& S0, const CoefT<R>& c0, const Batch<R>& b, bool sx,
                        bool sy, bool bed, cudaStream_t st, Trace* tr) {
  launch_half_x(S0, c0, sx, st, tr, b);
  if (sx) launch_sediment(S0, c0, true, false, st, tr, b);
  launch_half_y(S0, c0, sy, st, tr, b, sy && bed);
  if (sy) launch_sediment(S0, c0, false, bed, st, tr, b);
}

template <class R>
int upload_batch(HydistEnsemble* e, StateT<R> HydistHandle::*sm, CoefT<R> HydistHandle::*cm) {
  const int n = (int)e->m.size();
  std::vector<StateT<R>> S(n);
  std::vector<CoefT<R>> C(n);
  for (int i = 0; i < n; ++i) {
    S[i] = e->m[i]->*sm;
    C[i] = e->m[i]->*cm;
  }
  CK(cudaMalloc(&e->bS, n * sizeof(StateT<R>)));
  CK(cudaMalloc(&e->bC, n * sizeof(CoefT<R>)));
  CK(cudaMemcpy(e->bS, S.data(), n * sizeof(StateT<R>), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(e->bC, C.data(), n * sizeof(CoefT<R>), cudaMemcpyHostToDevice));
  return HYDIST_OK;
}

}  // namespace

extern "C" {

int hydist_ensemble_create(HydistHandle* const* members, int32_t n, HydistEnsemble** out) {
  if (!members || !out || n < 1) return fail(HYDIST_ERR_ARG, "null argument or empty ensemble");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!members[i]) return fail(HYDIST_ERR_ARG, "null member");
    if (members[i]->device != members[0]->device)
      return fail(HYDIST_ERR_ARG, "members must be on one device");
    if (members[i]->next_half) return fail(HYDIST_ERR_STATE, "a member has a half-step pending");
    for (int j = 0; j < i; ++j)
      if (members[j] == members[i]) return fail(HYDIST_ERR_ARG, "a member appears twice");
  }
  auto* e = new HydistEnsemble();
  e->device = members[0]->device;
  e->m.assign(members, members + n);
  int rc = [&]() -> int {
    CK(cudaSetDevice(e->device));
    CK(cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming));
    e->join.resize(n);
    for (auto& ev : e->join) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    e->uniform = true;
    for (int i = 1; i < n; ++i) e->uniform = e->uniform && same_launches(members[0], members[i]);
    if (e->uniform) {
      if (members[0]->fp32) TRY(upload_batch<float>(e, &HydistHandle::Sf, &HydistHandle::cf));
      else TRY(upload_batch<double>(e, &HydistHandle::S, &HydistHandle::c));
      e->batched = true;
    }
    return HYDIST_OK;
  }();
  if (rc != HYDIST_OK) {
    hydist_ensemble_destroy(e);
    return rc;
  }
  *out = e;
  return HYDIST_OK;
}

int hydist_ensemble_destroy(HydistEnsemble* e) {
  if (!e) return HYDIST_OK;
  cudaSetDevice(e->device);
  if (e->origin) cudaStreamSynchronize(e->origin);
  for (auto& kv : e->graphs)
    if (kv.second.first) cudaGraphExecDestroy(kv.second.first);
  for (auto& ev : e->join)
    if (ev) cudaEventDestroy(ev);
  if (e->bS) cudaFree(e->bS);
  if (e->bC) cudaFree(e->bC);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->done) cudaEventDestroy(e->done);
  if (e->origin) cudaStreamDestroy(e->origin);
  delete e;
  return HYDIST_OK;
}

int hydist_ensemble_step(HydistEnsemble* e, int32_t nsteps) {
  if (!e) return fail(HYDIST_ERR_ARG, "null ensemble");
  if (nsteps < 0) return fail(HYDIST_ERR_ARG, "negative step count");
  const int n = (int)e->m.size();
  CK(cudaSetDevice(e->device));
  for (HydistHandle* h : e->m) {
    if (h->next_half) return fail(HYDIST_ERR_STATE, "a member has a half-step pending");
    TRY(check_horizon(h, nsteps));
  }
  if (nsteps == 0) return HYDIST_OK;
  // the graph runs after each member's earlier work ...
  for (int i = 0; i < n; ++i) {
    CK(cudaEventRecord(e->join[i], e->m[i]->stream));
    CK(cudaStreamWaitEvent(e->origin, e->join[i], 0));
  }
  std::vector<unsigned char> key(3 * n);
  for (int k = 0; k < nsteps; ++k) {
    for (int i = 0; i < n; ++i) {
      const HydistHandle* h = e->m[i];
      const double t1 = h->t + 0.5 * h->c.dT, t2 = t1 + h->c.dT * 0.5;
      key[3 * i] = t1 >= h->o.sediment_start;
      key[3 * i + 1] = t2 >= h->o.sediment_start;
      key[3 * i + 2] = bed_on(h, t2);
    }
    // all members in the same sediment phase: one launch per kernel for the
    // batch (the graph's key is that phase alone)
    bool same = e->batched;
    for (int i = 1; same && i < n; ++i)
      same = key[3 * i] == key[0] && key[3 * i + 1] == key[1] && key[3 * i + 2] == key[2];
    std::vector<unsigned char> gkey = same ? std::vector<unsigned char>{2, key[0], key[1], key[2]}
                                           : key;
    auto it = e->graphs.find(gkey);
    if (it == e->graphs.end()) {
      cudaGraph_t g = nullptr;
      long long launches = 0;
      CK(cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal));
      if (same) {
        HydistHandle* h0 = e->m[0];
        Trace tr;
        if (h0->fp32) {
          const Batch<float> b{static_cast<const StateT<float>*>(e->bS),
                               static_cast<const CoefT<float>*>(e->bC), n};
          enqueue_step_batch(h0->Sf, h0->cf, b, key[0], key[1], key[2], e->origin, &tr);
        } else {
          const Batch<double> b{static_cast<const State*>(e->bS),
                                static_cast<const Coef*>(e->bC), n};
          enqueue_step_batch(h0->S, h0->c, b, key[0], key[1], key[2], e->origin, &tr);
        }
        launches = tr.launches;
      } else {
        // one step of every member: fork from the origin stream onto the
        // members' streams, join back
        CK(cudaEventRecord(e->fork, e->origin));
        for (int i = 0; i < n; ++i) {
          HydistHandle* h = e->m[i];
          CK(cudaStreamWaitEvent(h->stream, e->fork, 0));
          Trace tr;
          enqueue_step(h, key[3 * i], key[3 * i + 1], key[3 * i + 2], &tr);
          launches += tr.launches;
          CK(cudaEventRecord(e->join[i], h->stream));
          CK(cudaStreamWaitEvent(e->origin, e->join[i], 0));
        }
      }
      CK(cudaStreamEndCapture(e->origin, &g));
      cudaGraphExec_t ex = nullptr;
      const cudaError_t err = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      CK(err);
      it = e->graphs.emplace(gkey, std::make_pair(ex, launches)).first;
    }
    CK(cudaGraphLaunch(it->second.first, e->origin));
    for (int i = 0; i < n; ++i) {
      HydistHandle* h = e->m[i];
      const double t1 = h->t + 0.5 * h->c.dT;
      h->t = t1 + h->c.dT * 0.5;
    }
    e->m[0]->trace.launches += it->second.second;  // counted once, on the first member
  }
  // ... and each member's later work runs after the graph
  CK(cudaEventRecord(e->done, e->origin));
  for (HydistHandle* h : e->m) CK(cudaStreamWaitEvent(h->stream, e->done, 0));
  return HYDIST_OK;
}

void* hydist_ensemble_stream(HydistEnsemble* e) { return e ? (void*)e->origin : nullptr; }

int hydist_ensemble_batched(HydistEnsemble* e, int32_t enable) {
  if (!e) return fail(HYDIST_ERR_ARG, "null ensemble");
  if (enable && !e->uniform)
    return fail(HYDIST_ERR_ARG, "the members differ in mesh size, form or launch options");
  e->batched = enable != 0;
  return HYDIST_OK;
}

int hydist_ensemble_sync(HydistEnsemble* e) {
  if (!e) return fail(HYDIST_ERR_ARG, "null ensemble");
  CK(cudaSetDevice(e->device));
  CK(cudaStreamSynchronize(e->origin));
  for (HydistHandle* h : e->m) TRY(check_device_err(h));
  return HYDIST_OK;
}

// ---- checkpoint / resume -------------------------------------------------
// File: a fixed header, then the fields that carry from step to step, each
// (N+3)*(M+3) FP64 in the HydistField order of kCheckpointFields, then the
// int32 mask. The segment tables are derived from the mask (rescanned on
// load), the boundary arrays and smoothing buffers are rewritten every
// half-step before they are read.
namespace {

const int kCheckpointFields[] = {
    HYDIST_FIELD_U,   HYDIST_FIELD_V,  HYDIST_FIELD_Z,    HYDIST_FIELD_TU,  HYDIST_FIELD_TV,
    HYDIST_FIELD_TZ,  HYDIST_FIELD_H_MOI, HYDIST_FIELD_HTDU, HYDIST_FIELD_HTDV, HYDIST_FIELD_FS,
    HYDIST_FIELD_TFS, HYDIST_FIELD_VTH, HYDIST_FIELD_KX,  HYDIST_FIELD_KY,  HYDIST_FIELD_DH,
    HYDIST_FIELD_QBX, HYDIST_FIELD_QBY};

struct CheckpointHeader {
  char magic[8];  // "HYDISTCK"
  int32_t version, M, N, nfields;
  double t;
  int32_t next_half, reserved;
};

}  // namespace

int hydist_checkpoint_save(HydistHandle* h, const char* path) {
  if (!h || !path) return fail(HYDIST_ERR_ARG, "null argument");
  if (h->next_half) return fail(HYDIST_ERR_STATE, "save between full steps");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  const size_t n = (size_t)h->S.W * h->S.H;
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(HYDIST_ERR_ARG, std::string("cannot open ") + path);
  CheckpointHeader hd{};
  std::memcpy(hd.magic, "HYDISTCK", 8);
  hd.version = 1;
  hd.M = h->S.M;
  hd.N = h->S.N;
  hd.nfields = (int32_t)(sizeof(kCheckpointFields) / sizeof(int));
  hd.t = h->t;
  hd.next_half = 0;
  bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1;
  std::vector<double> buf(n);
  for (int fid : kCheckpointFields) {
    if (!ok) break;
    ok = field_to_host(h, field_ref(h, fid), buf.data(), n) == HYDIST_OK &&
         std::fwrite(buf.data(), 8, n, f) == n;
  }
  std::vector<int32_t> mask(n);
  ok = ok && cudaMemcpy(mask.data(), h->S.khouot, n * 4, cudaMemcpyDeviceToHost) == cudaSuccess &&
       std::fwrite(mask.data(), 4, n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(HYDIST_ERR_CUDA, std::string("writing the checkpoint failed: ") + path);
  return HYDIST_OK;
}

int hydist_checkpoint_load(HydistHandle* h, const char* path) {
  if (!h || !path) return fail(HYDIST_ERR_ARG, "null argument");
  if (h->next_half) return fail(HYDIST_ERR_STATE, "load between full steps");
  CK(cudaSetDevice(h->device));
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(HYDIST_ERR_ARG, std::string("cannot open ") + path);
  CheckpointHeader hd{};
  const int nf = (int)(sizeof(kCheckpointFields) / sizeof(int));
  if (std::fread(&hd, sizeof(hd), 1, f) != 1 || std::memcmp(hd.magic, "HYDISTCK", 8) != 0 ||
      hd.version != 1 || hd.nfields != nf) {
    std::fclose(f);
    return fail(HYDIST_ERR_ARG, "not a checkpoint of this format");
  }
  if (hd.M != h->S.M || hd.N != h->S.N) {
    std::fclose(f);
    return fail(HYDIST_ERR_ARG, "the checkpoint is of another mesh size");
  }
  // the whole body is read and its size checked before anything is
  // uploaded, so a truncated or oversized file leaves the handle unchanged
  const size_t n = (size_t)h->S.W * h->S.H;
  std::vector<double> body((size_t)nf * n);
  std::vector<int32_t> mask(n);
  bool ok = std::fread(body.data(), 8, body.size(), f) == body.size() &&
            std::fread(mask.data(), 4, n, f) == n;
  char extra;
  ok = ok && std::fread(&extra, 1, 1, f) == 0 && std::feof(f);
  std::fclose(f);
  if (!ok)
    return fail(HYDIST_ERR_ARG, std::string("checkpoint size does not match header + ") +
                                    std::to_string(nf) + " fields + mask: " + path);
  CK(cudaStreamSynchronize(h->stream));
  for (int k = 0; k < nf; ++k)
    TRY(field_from_host(h, field_ref(h, kCheckpointFields[k]), body.data() + (size_t)k * n, n));
  CK(cudaMemcpy(h->S.khouot, mask.data(), n * 4, cudaMemcpyHostToDevice));
  // with the bed feedback, the bed follows from the initial bed and dH
  if (h->S.bed_fb) on_state(h, [&](auto& St, auto& Cf) { launch_bed_feedback(St, Cf, h->stream); });
  on_state(h, [&](auto& St, auto& Cf) { launch_scan_segments(St, Cf, false, h->stream); });
  CK(cudaGetLastError());
  h->t = hd.t;
  TRY(set_device_clock(h));
  return check_device_err(h);
}

int hydist_set_time(HydistHandle* h, double t) {
  if (!h) return fail(HYDIST_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  h->t = t;
  return set_device_clock(h);
}

int hydist_download(HydistHandle* h, int32_t field, void* host) {
  if (!h || !host) return fail(HYDIST_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  const size_t n = (size_t)h->S.W * h->S.H;
  if (field == HYDIST_FIELD_KHOUOT) {
    CK(cudaMemcpyAsync(host, h->S.khouot, n * 4, cudaMemcpyDeviceToHost, h->stream));
  } else {
    const FieldRef r = field_ref(h, field);
    if (!r.p) return fail(HYDIST_ERR_ARG, "unknown field");
    return field_to_host(h, r, static_cast<double*>(host), n);
  }
  CK(cudaStreamSynchronize(h->stream));
  return HYDIST_OK;
}

int hydist_upload(HydistHandle* h, int32_t field, const void* host) {
  if (!h || !host) return fail(HYDIST_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  const size_t n = (size_t)h->S.W * h->S.H;
  if (field == HYDIST_FIELD_KHOUOT) {
    CK(cudaMemcpyAsync(h->S.khouot, host, n * 4, cudaMemcpyHostToDevice, h->stream));
    on_state(h, [&](auto& St, auto& Cf) { launch_scan_segments(St, Cf, false, h->stream); });
    CK(cudaGetLastError());
  } else {
    const FieldRef r = field_ref(h, field);
    if (!r.p) return fail(HYDIST_ERR_ARG, "unknown field");
    return field_from_host(h, r, static_cast<const double*>(host), n);
  }
  CK(cudaStreamSynchronize(h->stream));
  return HYDIST_OK;
}

int hydist_mass(HydistHandle* h, double* volume) {
  if (!h || !volume) return fail(HYDIST_ERR_ARG, "null argument");
  CK(cudaSetDevice(h->device));
  k_mass<<<h->mass_blocks, 256, 0, h->stream>>>(h->S, h->mass_part, h->mass_done, h->mass_host_dev);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  *volume = *(volatile double*)h->mass_host * h->c.dX * h->c.dY;
  return HYDIST_OK;
}

void* hydist_stream(HydistHandle* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"
