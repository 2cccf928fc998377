// ref_driver.cu -- TEST INFRASTRUCTURE ONLY.
//
// Runs the unmodified reference time step (compiled from the reference's own
// sources) on a reference-format input directory and writes the state in
// full FP64 precision at chosen step counts, so that the CPU oracle can be
// checked against the reference itself. The set-up calls are the reference's
// public functions (loader.h, support_funcs.h, engine.h) in the order its
// main() uses them (main.cpp:138-309); the reference prints only 6 digits of
// its fields (loader.cpp:378-414), hence this driver.
//
// usage: hydist_ref_driver <input_dir/> <out_dir> <steps_csv> [key=value ...]
//   keys: sediment_start, bed_change_start, dX, dT, Toe, Tod, Mbochat, wss,
//         fs0 (binary float64 file of (N+3)*(M+3) initial concentration),
//         z0 (the same for the initial water level, loaded into z and t_z
//         before the set-up kernels, as a warm start would be),
//         ketdinh (0: non-cohesive source), kenhhepd / kenhhepng (the
//         narrow-channel options of main.cpp's -kd / -kn), Wind, huonggio,
//         CORIOLIS (Constant_Coeffs members; Windx / Windy derived as
//         Load_coeffs derives them, loader.cpp:81-82)
// Output: <out_dir>/state_<steps>.bin = int32 {N, M, steps, nfields},
//         double t, then nfields float64 arrays of (N+3)*(M+3):
//         u v z FS H_moi t_u t_v t_z Htdu Htdv khouot tFS VTH Kx Ky
//         (plus ubt, ubp padded... not written)
// stdout of the reference (it prints t every half-step) should be
// redirected by the caller.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.h"
#include "loader.h"
#include "support_funcs.h"

static void die(const char* m) {
  fprintf(stderr, "ref_driver: %s\n", m);
  exit(2);
}

static void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "ref_driver: %s: %s\n", what, cudaGetErrorString(e));
    exit(3);
  }
}

static void recompute_derived(Constant_Coeffs& c) {
  // the derived members Load_coeffs computes from dX, dY, dT (loader.cpp:9-17)
  c.dXbp = c.dX * c.dX;
  c.dX2 = 2 * c.dX;
  c.dYbp = c.dY * c.dY;
  c.dY2 = 2 * c.dY;
  c.dTchia2dX = c.dT / c.dX2;
  c.dTchia2dY = c.dT / c.dY2;
  c.HaiChiadT = 2.0 / c.dT;
}

int main(int argc, char** argv) {
  if (argc < 4) die("usage: hydist_ref_driver <input_dir/> <out_dir> <steps_csv> [k=v ...]");
  std::string dir = argv[1];
  std::string out = argv[2];
  std::vector<int> ckpts;
  {
    std::string s = argv[3];
    size_t p = 0;
    while (p < s.size()) {
      size_t q = s.find(',', p);
      if (q == std::string::npos) q = s.size();
      ckpts.push_back(atoi(s.substr(p, q - p).c_str()));
      p = q + 1;
    }
  }
  std::map<std::string, std::string> kv;
  for (int a = 4; a < argc; ++a) {
    std::string s = argv[a];
    size_t e = s.find('=');
    if (e != std::string::npos) kv[s.substr(0, e)] = s.substr(e + 1);
  }
  auto getd = [&](const char* k, double def) {
    return kv.count(k) ? atof(kv[k].c_str()) : def;
  };

  std::vector<DOUBLE> h, hsnham, VISCOIDX, Fw, FS, dH, bc_up, bc_down, bc_left, bc_right, CC_u,
      CC_d, CC_l, CC_r, u, v, z;
  std::vector<int> khouot, bienQ, boundary_type;
  int total_time = 0;
  // same argument order as main.cpp:138 (the reference's down/right series
  // therefore come from bienphai.txt / bienduoi.txt)
  std::pair<int, int> sz = load_inputs(dir, h, hsnham, VISCOIDX, Fw, bc_up, bc_down, bc_left,
                                       bc_right, CC_u, CC_d, CC_l, CC_r, bienQ, boundary_type,
                                       &total_time);
  const int N = sz.first - 3, M = sz.second - 3;
  if (N < 4 || M < 4) die("bad mesh");
  const size_t n = (size_t)(N + 3) * (M + 3);

  Host_arrays ha;
  ha.M = M;
  ha.N = N;
  ha.h = h;
  ha.hsnham = hsnham;
  ha.VISCOIDX = VISCOIDX;
  ha.Fw = Fw;
  ha.FS = FS;
  ha.dH = dH;
  ha.bc_up = bc_up;
  ha.bc_down = bc_down;
  ha.bc_left = bc_left;
  ha.bc_right = bc_right;
  ha.CC_u = CC_u;
  ha.CC_d = CC_d;
  ha.CC_l = CC_l;
  ha.CC_r = CC_r;
  ha.u = u;
  ha.v = v;
  ha.z = z;
  ha.khouot = khouot;
  ha.bienQ = bienQ;
  ha.boundary_type = boundary_type;

  Argument_Pointers* d_arg = nullptr;
  Array_Pointers* d_arr = nullptr;
  Argument_Pointers h_arg = attribute_arrays_memory_alloc(0, ha, &d_arg);
  // The scratch arrays of Array_Pointers are caller-owned. The reference's
  // supporting_arrays_alloc (loader.cpp:333-375) sizes SN as 20*max(M,N)
  // ints, but VZSolver_calculate_matrix_coeff writes SN[20*N + k] when row N
  // is wet (UVZSolver_multithread.cpp:468); that write lands on the next
  // allocation -- the device copy of Array_Pointers itself -- and corrupts
  // its first pointer. The a1..f5 arrays are also indexed past M*N+2max(M,N)
  // (:159-165, 228-234). The same arrays are allocated here with padding.
  Array_Pointers h_arr;
  {
    const size_t s1 = sizeof(DOUBLE) * ((size_t)(N + 3) * (M + 3) + 2 * std::max(M, N) + 64);
    const size_t s2 = sizeof(DOUBLE) * (2 * (size_t)(N + 3) * (M + 3) + 4 * std::max(M, N) + 64);
    DOUBLE** a1[] = {&h_arr.a1, &h_arr.b1, &h_arr.c1, &h_arr.d1, &h_arr.a2, &h_arr.c2,
                     &h_arr.d2, &h_arr.f1, &h_arr.f2, &h_arr.f3, &h_arr.f5};
    for (DOUBLE** p : a1) ck(cudaMalloc((void**)p, s1), "malloc scratch");
    DOUBLE** a2[] = {&h_arr.AA, &h_arr.BB, &h_arr.CC, &h_arr.DD,
                     &h_arr.Ap, &h_arr.Bp, &h_arr.ep, &h_arr.x};
    for (DOUBLE** p : a2) ck(cudaMalloc((void**)p, s2), "malloc scratch");
    ck(cudaMalloc((void**)&h_arr.SN, sizeof(int) * segment_limit * (std::max(M, N) + 8)),
       "malloc SN");
    ck(cudaMalloc((void**)&d_arr, sizeof(Array_Pointers)), "malloc arr");
    ck(cudaMemcpy(d_arr, &h_arr, sizeof(Array_Pointers), cudaMemcpyHostToDevice), "arr");
  }

  // The reference relies on freshly allocated device memory being zero
  // (loader.cpp:269-304); make that explicit.
  const size_t nb = n * sizeof(DOUBLE);
  DOUBLE* zf[] = {h_arg.u, h_arg.v, h_arg.z, h_arg.t_u, h_arg.t_v, h_arg.t_z, h_arg.Kx1,
                  h_arg.Ky1, h_arg.Htdu, h_arg.Htdv, h_arg.htaiz, h_arg.htaiz_bd, h_arg.H_moi,
                  h_arg.Tsxw, h_arg.Tsyw, h_arg.VTH, h_arg.Qbx, h_arg.Qby, h_arg.FS, h_arg.tFS,
                  h_arg.Kx, h_arg.Ky, h_arg.dH};
  for (DOUBLE* p : zf) ck(cudaMemset(p, 0, nb), "memset");
  ck(cudaMemset(h_arg.khouot, 0, n * sizeof(int)), "memset");
  ck(cudaMemset(h_arg.ubt, 0, sizeof(DOUBLE) * (M + 2)), "memset");
  ck(cudaMemset(h_arg.ubp, 0, sizeof(DOUBLE) * (M + 2)), "memset");
  ck(cudaMemset(h_arg.vbt, 0, sizeof(DOUBLE) * (N + 2)), "memset");
  ck(cudaMemset(h_arg.vbd, 0, sizeof(DOUBLE) * (N + 2)), "memset");
  ck(cudaMemset(h_arg.hi, 0, sizeof(DOUBLE) * (2 * (M + N + 6))), "memset");
  {
    const size_t s1 = sizeof(DOUBLE) * ((size_t)(N + 3) * (M + 3) + 2 * std::max(M, N) + 64);
    const size_t s2 = sizeof(DOUBLE) * (2 * (size_t)(N + 3) * (M + 3) + 4 * std::max(M, N) + 64);
    DOUBLE* a1[] = {h_arr.a1, h_arr.b1, h_arr.c1, h_arr.d1, h_arr.a2, h_arr.c2,
                    h_arr.d2, h_arr.f1, h_arr.f2, h_arr.f3, h_arr.f5};
    for (DOUBLE* p : a1) ck(cudaMemset(p, 0, s1), "memset");
    DOUBLE* a2[] = {h_arr.AA, h_arr.BB, h_arr.CC, h_arr.DD, h_arr.Ap, h_arr.Bp, h_arr.ep, h_arr.x};
    for (DOUBLE* p : a2) ck(cudaMemset(p, 0, s2), "memset");
    ck(cudaMemset(h_arr.SN, 0, sizeof(int) * segment_limit * (std::max(M, N) + 8)), "memset");
  }
  if (kv.count("z0")) {
    std::vector<double> z0(n);
    FILE* f = fopen(kv["z0"].c_str(), "rb");
    if (!f || fread(z0.data(), sizeof(double), n, f) != n) die("cannot read z0");
    fclose(f);
    ck(cudaMemcpy(h_arg.z, z0.data(), nb, cudaMemcpyHostToDevice), "z0");
    ck(cudaMemcpy(h_arg.t_z, z0.data(), nb, cudaMemcpyHostToDevice), "z0");
  }
  if (kv.count("fs0")) {
    std::vector<double> fs0(n);
    FILE* f = fopen(kv["fs0"].c_str(), "rb");
    if (!f || fread(fs0.data(), sizeof(double), n, f) != n) die("cannot read fs0");
    fclose(f);
    ck(cudaMemcpy(h_arg.FS, fs0.data(), nb, cudaMemcpyHostToDevice), "fs0");
    ck(cudaMemcpy(h_arg.tFS, fs0.data(), nb, cudaMemcpyHostToDevice), "fs0");
  }

  Constant_Coeffs hc, *dc = nullptr;
  Load_coeffs(hc);
  if (kv.count("dX")) {
    hc.dX = hc.dY = getd("dX", hc.dX);
  }
  if (kv.count("dT")) hc.dT = getd("dT", hc.dT);
  recompute_derived(hc);
  if (kv.count("Toe")) hc.Toe = getd("Toe", hc.Toe);
  if (kv.count("Tod")) hc.Tod = getd("Tod", hc.Tod);
  if (kv.count("Mbochat")) hc.Mbochat = getd("Mbochat", hc.Mbochat);
  if (kv.count("wss")) hc.wss = getd("wss", hc.wss);
  if (kv.count("CORIOLIS")) hc.CORIOLIS_FORCE = getd("CORIOLIS", hc.CORIOLIS_FORCE);
  if (kv.count("Wind") || kv.count("huonggio")) {
    hc.Wind = getd("Wind", hc.Wind);
    hc.huonggio = getd("huonggio", hc.huonggio);
    const double W = hc.Wind, aW = W < 0 ? -W : W;
    hc.Windx = 0.0013 * (0.00075 + 0.000067 * aW) * aW * W * cos(hc.huonggio * (PI / 180));
    hc.Windy = 0.0013 * (0.00075 + 0.000067 * aW) * aW * W * sin(hc.huonggio * (PI / 180));
  }
  ck(cudaMalloc((void**)&dc, sizeof(Constant_Coeffs)), "malloc coeffs");
  ck(cudaMemcpy(dc, &hc, sizeof(Constant_Coeffs), cudaMemcpyHostToDevice), "coeffs");

  // set-up kernels with the launch shapes of main.cpp:258-299
  dim3 block_2d(std::min(32, M + 3), 1, 1);
  dim3 grid_2d((M + 3) / std::min(32, M + 3) + 1, N + 3, 1);
  Onetime_init<<<grid_2d, block_2d>>>(d_arg, dc);
  synch_and_check();
  Find_Calculation_limits_Horizontal<<<dim3(1, N, 1), 32>>>(d_arg, dc);
  Find_Calculation_limits_Vertical<<<dim3(1, M, 1), 32>>>(d_arg, dc);
  Htuongdoi<<<grid_2d, block_2d>>>(d_arg);
  synch_and_check();
  preprocess_data<<<1, 32>>>(d_arg, dc);
  synch_and_check();

  const double sed = getd("sediment_start", 1e12);
  const double bcs = getd("bed_change_start", 1e12);
  const bool cohesive = getd("ketdinh", 1) != 0;
  const bool kd = getd("kenhhepd", 0) != 0, kn = getd("kenhhepng", 0) != 0;
  // Options(Tmax, t_start, interval, sediment_start, bed_change_start,
  // cohesive, kenhng, kenhd, debug, plot), engine.h:25-35
  Options ops(0.0, 0.0, 1 << 30, sed, bcs, cohesive, kn, kd, false, false);
  ops.M = M;
  ops.N = N;
  ops.total_time = total_time;

  std::vector<double> buf(n);
  std::vector<int> ibuf(n);
  int done = 0;
  double t = 0.0;
  for (int target : ckpts) {
    if (target > done) {
      ops.t_start = t;
      ops.Tmax = t + (target - done) * hc.dT;
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      cudaEventRecord(e0);
      Hydraulic_Calculation(hc.dT, hc.NANGDAY, d_arg, d_arr, dc, h_arg, ops);
      cudaEventRecord(e1);
      synch_and_check();
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      // the reference's own time step, device-timed (it synchronises after
      // every kernel, so this is also its wall time)
      fprintf(stderr, "ref_driver: Hydraulic_Calculation steps %d..%d: %.3f ms\n", done, target, ms);
      t = ops.Tmax;
      done = target;
    }
    std::string fn = out + "/state_" + std::to_string(target) + ".bin";
    FILE* f = fopen(fn.c_str(), "wb");
    if (!f) die("cannot open output");
    DOUBLE* fields[] = {h_arg.u,    h_arg.v,    h_arg.z,   h_arg.FS,  h_arg.H_moi,
                        h_arg.t_u,  h_arg.t_v,  h_arg.t_z, h_arg.Htdu, h_arg.Htdv,
                        nullptr,    h_arg.tFS,  h_arg.VTH, h_arg.Kx,  h_arg.Ky};
    int hdr[4] = {N, M, target, (int)(sizeof(fields) / sizeof(fields[0]))};
    fwrite(hdr, sizeof(int), 4, f);
    fwrite(&t, sizeof(double), 1, f);
    for (DOUBLE* p : fields) {
      if (p == nullptr) {
        ck(cudaMemcpy(ibuf.data(), h_arg.khouot, n * sizeof(int), cudaMemcpyDeviceToHost), "d2h");
        for (size_t k = 0; k < n; ++k) buf[k] = ibuf[k];
      } else {
        ck(cudaMemcpy(buf.data(), p, nb, cudaMemcpyDeviceToHost), "d2h");
      }
      fwrite(buf.data(), sizeof(double), n, f);
    }
    fclose(f);
    fprintf(stderr, "ref_driver: wrote %s (t=%.1f)\n", fn.c_str(), t);
  }
  return 0;
}
