// sweep.cu -- the hydraulic ADI line sweeps on the partitioned line solver.
//
// HydroGen<0> is the x sweep (UZ half-step: lines are columns j, cells run
// along i, unknowns z_i and u_i interleaved); HydroGen<1> is the y sweep (VZ
// half-step: lines are rows i, cells along j, unknowns z_j and v_j). Both
// generate the reference's tridiagonal rows on the fly (assembly.cuh) and
// write the extraction of UZSolver_extract_solution / VZSolver_extract_
// solution (UVZSolver_multithread.cpp:472-603) directly from the solution.
#include "assembly.cuh"
#include "common.cuh"

#include "hydro.cuh"
#include "linesolve.cuh"
#include "sediment_cell.cuh"

namespace hyd {

// chunks per line: as many as keep at least `min_cells` cells per chunk (of
// 128, 64, 32, 16, 4 or 1), so that no chunk of a short line is empty or
// holds its separator alone
int line_chunks(int ncells, int min_cells) {
  int P = 128;
  while (P > 1 && ncells < P * min_cells) P >>= 1;
  if (P == 8) P = 4;
  if (P == 2) P = 1;
  return P;
}

// REF: refine each line solve once with an FP64 residual (FP32 forms)
template <int DIR, class R, bool REF = false>
struct HydroGen {
  using Real = R;
  static constexpr bool REFINE = REF;
  // the rows are generated from the stencils: the refinement keeps them
  static constexpr bool ROWS_AGAIN = false;
  static constexpr int SCRATCH_ARRAYS = REFINE ? 7 : 3;
  static constexpr int UPC = 2;
  static constexpr int DIRECTION = DIR;
  // x sweeps (columns, 4 adjacent per warp) run faster with two CTAs per SM
  // despite the register cap, and so do the FP32 y sweeps; the FP64 and the
  // refined FP32 y sweeps slower
  static constexpr int MIN_BLOCKS = (DIR == 0 || (sizeof(R) == 4 && !REF)) ? 2 : 1;
  StateT<R> S;
  CoefT<R> c;
  R* scratch;
  R f4;
  // lines lp0 .. lp0 + nl - 1: columns 2..M (x) / rows 2..N (y), or the
  // narrow-channel ranges (StateT::x_lo, x_hi, y_lo)
  int lp0, nl;

  __host__ __device__ void bind(const StateT<R>& s, const CoefT<R>& cc) {
    S = s;
    c = cc;
    f4 = DIR == 0 ? 2 * cc.g * cc.dTchia2dX : 2 * cc.g * cc.dTchia2dY;
  }
  __device__ int lines() const { return nl; }
  __device__ int cells_per_line() const { return DIR == 0 ? S.N - 1 : S.M - 1; }
  __device__ int unknowns_per_line() const { return 2 * cells_per_line(); }
  __device__ int end_pos() const { return DIR == 0 ? S.N : S.M; }
  // field index of position p on line position lp
  __device__ int at(int lp, int p) const { return DIR == 0 ? p * S.W + lp : lp * S.W + p; }
  // the preindex values of a cell, from its stencil (computed where the
  // walker reaches the cell: a separate per-cell pass writing them to HBM
  // ahead of the sweep costs more in traffic and a launch than it saves)
  __device__ PreT<R> pre(int lp, int p) const {
    return DIR == 0 ? pre_x(S, c, p, lp) : pre_y(S, c, lp, p);
  }
  __device__ R* vel() const { return DIR == 0 ? S.tu : S.tv; }
  // the VZ extraction reaches columns j <= N only (UVZSolver_multithread.cpp:851)
  __device__ bool extract_ok(int p) const { return DIR == 0 ? true : p <= S.N; }

  __device__ void load_segment(LineSeg& LS, int line, int s) const {
    const bool ok = line < lines();
    const int lp = line + lp0;
    if (s == SEG) {
      LS.nseg = ok ? (DIR == 0 ? S.mocj[lp] : S.moci[lp]) : 0;
      return;
    }
    if (!ok) return;
    const int n = DIR == 0 ? S.mocj[lp] : S.moci[lp];
    if (s >= n) return;
    const int w = S.W;
    SegD& d = LS.s[s];
    int first, last;
    bool br1, br2;
    bool q1, q2;
    if (DIR == 0) {
      first = S.dauj[lp * SEG + s];
      last = S.cuoij[lp * SEG + s];
      // locate_segment_u (support_funcs.cpp:845-851)
      br1 = (first > 2) || ((first == 2) && ((S.h[1 * w + lp] + S.h[1 * w + lp - 1]) * 0.5 == c.NANGDAY));
      br2 = (last < S.N) || ((last == S.N) && ((S.h[S.N * w + lp] + S.h[S.N * w + lp - 1]) * 0.5 == c.NANGDAY));
      q1 = S.bienQ[2] != 0;
      q2 = S.bienQ[3] != 0;
    } else {
      first = S.daui[lp * SEG + s];
      last = S.cuoii[lp * SEG + s];
      // locate_segment_v (support_funcs.cpp:823-826)
      br1 = (first > 2) || ((first == 2) && ((S.h[lp * w + first - 1] + S.h[(lp - 1) * w + first - 1]) * 0.5 == c.NANGDAY));
      br2 = (last < S.M) || ((last == S.M) && ((S.h[lp * w + last] + S.h[(lp - 1) * w + last]) * 0.5 == c.NANGDAY));
      q1 = S.bienQ[1] != 0;
      q2 = S.bienQ[0] != 0;
    }
    const LineSys L = line_sys(first, last, br1, br2, q1, q2, end_pos());
    d.first = first;
    d.last = last;
    d.off = L.off;
    d.rend = L.off + L.sn;
    d.br1 = br1;
    d.br2 = br2;
    d.ran = L.ran;
    d.qfirst = L.qfirst;
    d.last_kind = (unsigned char)L.last_kind;
    d.xq_first = q1;
    d.xq_last = q2;
  }

  // Generates the rows of the line system cell by cell (two unknowns per cell).
  struct Walker {
    int lp, si, pos, prev;
    bool in;
    PreT<R> Pc, Pn;
    MomT<R> Mi;
    __device__ void init(const HydroGen& G, const LineSeg& LS, int line, int c0) {
      lp = line + G.lp0;
      si = 0;
      prev = -10;
      in = false;
    }
    __device__ void cell(const HydroGen& G, const LineSeg& LS, int c) {
      pos = c + 2;
      while (si < LS.nseg && LS.s[si].last < pos) ++si;
      in = si < LS.nseg && LS.s[si].first <= pos;
      if (!in) {
        prev = -10;
        return;
      }
      const SegD& d = LS.s[si];
      if (prev == pos - 1 && pos > d.first) Pc = Pn;
      else Pc = G.pre(lp, pos);
      if (pos + 1 <= d.last) Pn = G.pre(lp, pos + 1);
      else Pn = Pc;
      if (pos <= d.last - 1 || pos == d.first) Mi = abcd(Pc, Pn, pos, d.first, d.last, G.f4, d.br1, d.br2);
      else Mi = MomT<R>{0, 0, 0, 0};
      prev = pos;
    }
    __device__ void row(const HydroGen& G, const LineSeg& LS, int e, R& A, R& B, R& C,
                        R& D) const {
      if (!in) {
        A = 0; B = 1; C = 0; D = 0;
        return;
      }
      G.rows_in(LS.s[si], lp, pos, Pc, Pn, Mi, e, A, B, C, D);
    }
  };

  // Row 2*pos + e of the line system at line position lp, for a cell pos of
  // segment d with its preindex values Pc, those of the next cell Pn (Pc at
  // the segment's last cell) and its momentum coefficients Mi.
  __device__ void rows_in(const SegD& d, int lp, int pos, const PreT<R>& Pc, const PreT<R>& Pn,
                          const MomT<R>& Mi, int e, R& A, R& B, R& C, R& D) const {
    const int r = 2 * pos + e;
    if (r < d.off || r > d.rend) {
      A = 0; B = 1; C = 0; D = 0;
      return;
    }
    const bool even = (r & 1) == 0;
    if ((bool)d.ran == even) {
      const PreT<R>& P = d.ran ? Pc : Pn;
      A = P.a2; B = 1; C = P.c2; D = P.d2;
    } else {
      A = Mi.a1; B = Mi.b1; C = Mi.c1; D = Mi.d1;
    }
    if (r == d.off) {
      if (d.ran) {
        if (d.qfirst) {
          const R ub = DIR == 0 ? S.ubt[lp] : S.vbd[lp];
          D = Pc.d2 - Pc.a2 * ub;
        } else {
          D = Pc.d2;
        }
      } else {
        const R TZ_l = R(S.tz[at(lp, d.first)]);
        D = Mi.d1 - Mi.a1 * TZ_l;
      }
      A = 0;  // the system starts here
    }
    if (r == d.rend) {
      const PreT<R>& PL = (pos == d.last) ? Pc : Pn;
      if (d.last_kind == 1) {
        const R ub = DIR == 0 ? S.ubp[lp] : S.vbt[lp];
        A = PL.a2; B = 1; D = PL.d2 - PL.c2 * ub;
      } else if (d.last_kind == 2) {
        const R TZ_r = R(S.tz[at(lp, d.last)]);
        A = Mi.a1; B = Mi.b1; D = Mi.d1 - Mi.c1 * TZ_r;
      } else {
        A = PL.a2; B = 1; D = PL.d2;
      }
      C = 0;  // and ends here
    }
  }

  // (the refinement reads the stored rows: no cursor over them)
  struct RowCursor {
    __device__ void init(const HydroGen&, const LineSeg&, int) {}
    __device__ void row(const HydroGen&, const LineSeg&, int, R&, R&, R&, R&) {}
  };

  // Writes each solved unknown to t_z / t_u (t_v) as the extraction does.
  // FWD: the unknowns come in increasing order (init_fwd), else decreasing.
  struct Emitter {
    int lp, si;
    __device__ void init(const HydroGen& G, const LineSeg& LS, int line) {
      lp = line + G.lp0;
      si = LS.nseg - 1;
    }
    __device__ void init_fwd(const HydroGen& G, const LineSeg& LS, int line) {
      lp = line + G.lp0;
      si = -1;
    }
    template <bool FWD = false>
    __device__ void emit(const HydroGen& G, const LineSeg& LS, double* xlast, int q, double x) {
      const int r = q + 4, pos = r >> 1;
      if constexpr (FWD) {
        while (si + 1 < LS.nseg && LS.s[si + 1].first <= pos) ++si;
      } else {
        while (si >= 0 && LS.s[si].first > pos) --si;
      }
      if (si < 0) return;
      G.store_in(LS.s[si], xlast + si, lp, q, x);
    }
  };

  // The extraction of unknown q (row q + 4) of segment d on line position
  // lp; the segment's last row also goes to *xl for the end fix-up.
  __device__ void store_in(const SegD& d, double* xl, int lp, int q, double x) const {
    const int r = q + 4, pos = r >> 1;
    if (pos > d.last || r < d.off || r > d.rend) return;
    if (r == d.rend) *xl = x;
    R* v = vel_ptr();
    if (d.ran) {
      const int i = r >> 1;
      if (i < d.last && extract_ok(i)) {
        if (r & 1) v[at(lp, i)] = x;
        else S.tz[at(lp, i)] = x;
      }
    } else {
      if (r == 2 * d.first) {
        if (extract_ok(d.first)) v[at(lp, d.first)] = x;
      } else {
        const int i = (r + 1) >> 1;
        if (i > d.first && i < d.last && extract_ok(i)) {
          if (r & 1) S.tz[at(lp, i)] = x;
          else v[at(lp, i)] = x;
        }
      }
    }
  }

  // Segment ends (_uzSolver_extract_solution :558-601 / _vzSolver_ :488-536).
  __device__ void fixup(const LineSeg& LS, const double* xlast, int line, int s) const {
    const SegD& d = LS.s[s];
    const int lp = line + lp0, first = d.first, last = d.last;
    R* vel = vel_ptr();
    double* tz = S.tz;
    if (first < last && extract_ok(first)) {
      if (d.br1) {
        vel[at(lp, first - 1)] = 0;
      } else if (d.xq_first && first == 2) {
        vel[at(lp, first - 1)] = DIR == 0 ? S.ubt[lp] : S.vbd[lp];
      } else {
        const PreT<R> Pf = pre(lp, first);
        vel[at(lp, first - 1)] = (Pf.d2 - tz[at(lp, first)] - Pf.c2 * vel[at(lp, first)]) / Pf.a2;
      }
    }
    if (!extract_ok(last)) return;
    const double xl = (d.rend >= d.off) ? xlast[s] : 0.0;
    if (d.br2) {
      vel[at(lp, last)] = 0;
      tz[at(lp, last)] = xl;
    } else if (d.xq_last && last == end_pos()) {
      vel[at(lp, last)] = DIR == 0 ? S.ubp[lp] : S.vbt[lp];
      tz[at(lp, last)] = xl;
    } else {
      const PreT<R> Pl = pre(lp, last);
      vel[at(lp, last)] = (Pl.d2 - Pl.a2 * vel[at(lp, last - 1)] - tz[at(lp, last)]) / Pl.c2;
    }
  }
  __device__ R* vel_ptr() const { return DIR == 0 ? S.tu : S.tv; }
};

// the kernel's shared-memory limit, raised once per device
template <class Gen, int P, int L>
static size_t prepare(int dev) {
  const size_t smem = line_smem<typename Gen::Real, P, L>(Gen::REFINE);
  static bool attr[64] = {};
  if (dev < 64 && !attr[dev]) {
    cudaFuncSetAttribute(k_line_solve<Gen, P, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    attr[dev] = true;
  }
  return smem;
}

template <class Gen, int P, int L = LPB>
static void launch_gen(const Gen& G, cudaStream_t st, int grid, int line0, int ngroups,
                       const Batch<typename Gen::Real>& b = {}, int gpm = 0) {
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t smem = prepare<Gen, P, L>(dev);
  if (b.n > 0) {
    static bool attr[64] = {};
    if (dev < 64 && !attr[dev]) {
      cudaFuncSetAttribute(k_line_solve<Gen, P, L, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      attr[dev] = true;
    }
    k_line_solve<Gen, P, L, 1><<<grid, L * P, smem, st>>>(G, line0, ngroups, b, gpm);
  } else {
    k_line_solve<Gen, P, L><<<grid, L * P, smem, st>>>(G, line0, ngroups, b, 0);
  }
}

template <class Gen>
static void launch_any(const Gen& G, int P, cudaStream_t st, int grid, int line0, int ngroups,
                       const Batch<typename Gen::Real>& b = {}, int gpm = 0) {
  if (P == 128) launch_gen<Gen, 128>(G, st, grid, line0, ngroups, b, gpm);
  else if (P == 64) launch_gen<Gen, 64>(G, st, grid, line0, ngroups, b, gpm);
  else if (P == 32) launch_gen<Gen, 32>(G, st, grid, line0, ngroups, b, gpm);
  else if (P == 16) launch_gen<Gen, 16>(G, st, grid, line0, ngroups, b, gpm);
  else if (P == 4) launch_gen<Gen, 4>(G, st, grid, line0, ngroups, b, gpm);
  else launch_gen<Gen, 1>(G, st, grid, line0, ngroups, b, gpm);
}

// CTAs of the 128-chunk solver resident on the device at once (queried once
// per device)
template <class Gen>
static int resident_slots() {
  static int slots[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return 0;
  if (!slots[dev]) {
    const size_t smem = prepare<Gen, 128, LPB>(dev);
    int per_sm = 0, nsm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_line_solve<Gen, 128, LPB>, LPB * 128,
                                                  smem);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    slots[dev] = per_sm * nsm;
  }
  return slots[dev];
}

// Launches a sweep over `lines` lines and returns the number of launches.
// In a row sweep whose last round of 4-line groups would leave more than
// half of the resident CTAs idle (2047 rows on 148 one-CTA SMs: 68 of 512
// groups), that remainder runs as a second launch of 2-line groups with 256
// chunks per line, half the chain per thread, on every SM.
//
// With a batch, one launch walks the line groups of every member (the
// persistent grid takes them in member order).
template <class Gen>
static int launch_lines(const Gen& G, int P, int lines, int lslots, cudaStream_t st,
                        const Batch<typename Gen::Real>& b = {}) {
  if constexpr (Gen::DIRECTION == 1 && Gen::UPC == 2 && !Gen::REFINE &&
                sizeof(typename Gen::Real) == 4) {
    if (P == 128) {
      // the FP32 hydraulic row sweep: groups of 8 rows, one 1024-thread CTA
      // per SM (its 64 registers as at two 512-thread CTAs): 0.130 -> 0.121
      // ms on 2048x1024 (the FP64 one, capped from 102 registers, 0.247
      // against 0.172: it keeps 4-row groups)
      const int g8 = cdiv(lines, XPB);
      const long long total = (long long)g8 * std::max(b.n, 1);
      launch_gen<Gen, 128, XPB>(G, st, (int)std::min<long long>(total, lslots / 2), 0, (int)total,
                                b, b.n > 0 ? g8 : 0);
      return 1;
    }
  }
  if constexpr (Gen::DIRECTION == 1 && Gen::UPC == 2 && Gen::REFINE) {
    if (P == 128 && b.n == 0) {
      // the refined hydraulic row sweep: groups of 8 rows of 64 chunks (one
      // 512-thread CTA per SM): 0.210 -> 0.204 ms on 2048x1024 (the FP64 and
      // FP32 ones slower that way: 0.231 / 0.153 against 0.173 / 0.131 ms)
      const int g8 = cdiv(lines, XPB);
      launch_gen<Gen, 64, XPB>(G, st, std::min(g8, lslots / 2), 0, g8);
      return 1;
    }
  }
  if constexpr (Gen::DIRECTION == 1) {
    if (P == 64 || (P == 128 && Gen::UPC == 1 && sizeof(typename Gen::Real) == 4)) {
      // row sweeps of 64 chunks (rows of 256 to 511 cells), and the FP32
      // concentration row sweeps of 128: groups of 8 adjacent rows (their
      // stencil rows shared through L1 by twice as many lines). The
      // 64-member ensemble of 1024x512 in FP32 with refinement: 13.64 ->
      // 12.63 ms per step (FP64 unchanged); the concentration y sweep of
      // 2048x1024 0.122 -> 0.108 ms refined, 0.087 -> 0.079 ms in FP32 (the
      // FP64 one 3 us slower, so it keeps 4-row groups). A group's scratch
      // slot is two 4-line slots.
      const int g8 = cdiv(lines, XPB);
      const long long total = (long long)g8 * std::max(b.n, 1);
      const int grid = (int)std::min<long long>(total, lslots / 2);
      if (P == 64) {
        launch_gen<Gen, 64, XPB>(G, st, grid, 0, (int)total, b, b.n > 0 ? g8 : 0);
      } else if constexpr (Gen::UPC == 1 && sizeof(typename Gen::Real) == 4) {
        launch_gen<Gen, 128, XPB>(G, st, grid, 0, (int)total, b, b.n > 0 ? g8 : 0);
      }
      return 1;
    }
  }
  if constexpr (Gen::DIRECTION == 0 && Gen::REFINE) {
    if (P == 64) {
      // the refined column sweeps of 64 chunks (columns of 256 to 511
      // cells) in groups of 8 columns: a 512x256 step 0.185 -> 0.178 ms,
      // 8 of them batched 0.576 -> 0.537 ms (the FP64 ones 3% slower that
      // way alone, unchanged batched: they keep groups of 4)
      const int g8 = cdiv(lines, XPB);
      const long long total = (long long)g8 * std::max(b.n, 1);
      launch_gen<Gen, 64, XPB>(G, st, (int)std::min<long long>(total, lslots / 2), 0, (int)total, b,
                               b.n > 0 ? g8 : 0);
      return 1;
    }
  }
  if constexpr (Gen::DIRECTION == 0) {
    if (P == 128) {
      // column sweeps of 128 chunks: groups of 8 adjacent columns, one CTA
      // of 1024 threads per SM (a warp's loads cover 64 contiguous bytes of
      // each of 4 chunk rows; a group's scratch slot is two of the 4-line
      // slots): 0.169 -> 0.153 ms for the FP64 hydraulic x sweep of
      // 2048x1024, 0.216 -> 0.154 ms refined in FP32
      const int g8 = cdiv(lines, XPB);
      if (b.n > 0) {
        const long long total = (long long)g8 * b.n;
        launch_gen<Gen, 128, XPB>(G, st, (int)std::min<long long>(total, lslots / 2), 0, (int)total,
                                  b, g8);
      } else {
        launch_gen<Gen, 128, XPB>(G, st, std::min(g8, lslots / 2), 0, g8);
      }
      return 1;
    }
  }
  const int groups = cdiv(lines, LPB);
  if (b.n > 0) {
    const long long total = (long long)groups * b.n;
    launch_any(G, P, st, (int)std::min<long long>(total, lslots), 0, (int)total, b, groups);
    return 1;
  }
  if constexpr (Gen::DIRECTION == 1) {
    if (P == 128) {
      const int slots = std::min(resident_slots<Gen>(), lslots);
      const int full = slots > 0 ? groups / slots : 0;
      const int rem = groups - full * slots;
      if (full >= 1 && rem > 0 && 2 * rem <= slots) {
        launch_gen<Gen, 128>(G, st, slots, 0, full * slots);
        const int line0 = full * slots * LPB;
        const int g2 = cdiv(lines - line0, 2);
        launch_gen<Gen, 256, 2>(G, st, std::min(g2, lslots), line0, g2);
        return 2;
      }
    }
  }
  launch_any(G, P, st, std::min(groups, lslots), 0, groups);
  return 1;
}

// Scratch slots for a sweep of lines of `unknowns` unknowns in P chunks:
// the scratch holds StateT::lslots slots of lines of 2*max(M, N) unknowns,
// so a sweep of shorter lines has proportionally more. Only the solvers of
// fewer than 128 chunks (smaller CTAs, more of them resident per SM) use
// them: their grid may then exceed the CTAs resident at once, the extra
// CTAs starting as earlier ones finish. (For the 128-chunk solvers the
// persistent grid of lslots CTAs measured as fast or faster.)
template <class R>
static int sweep_slots(const StateT<R>& S, int unknowns, int P) {
  if (P >= 128) return S.lslots;
  const int umax = 2 * std::max(S.M, S.N);
  return S.lslots * std::max(1, umax / std::max(unknowns, 1));
}

template <int DIR, class R, bool REF>
static int launch_dir(const StateT<R>& S, const CoefT<R>& c, cudaStream_t st, int P,
                      const Batch<R>& b) {
  HydroGen<DIR, R, REF> G;
  G.bind(S, c);
  G.scratch = S.lscratch;
  G.lp0 = DIR == 0 ? S.x_lo : S.y_lo;
  G.nl = DIR == 0 ? S.x_hi - S.x_lo + 1 : S.N - S.y_lo + 1;
  if (G.nl <= 0) return 0;
  const int ncells = DIR == 0 ? S.N - 1 : S.M - 1;
  return launch_lines(G, P, G.nl, sweep_slots(S, 2 * ncells, P), st, b);
}

// ---------------------------------------------------------------------
// Concentration sweeps: one unknown per cell, cells first+1..last-1 of each
// wet segment of at least three cells (Scan_FSj / Scan_FSi,
// sediment_transport.cpp:51-164, 204-313; extraction :167-201, 316-349).
// DIR 0: columns j = 3..M-1 along i; DIR 1: rows i = 3..N-1 along j.
template <int DIR, class R, bool REF = false>
struct FSGen {
  using Real = R;
  static constexpr bool REFINE = REF;
  // the rows are in StateT::pre (k_fs_rows): the refinement reads them again
  static constexpr bool ROWS_AGAIN = true;
  static constexpr int SCRATCH_ARRAYS = REFINE ? 4 : 3;
  static constexpr int UPC = 1;
  static constexpr int DIRECTION = DIR;
  // two CTAs per SM in both directions and precisions
  static constexpr int MIN_BLOCKS = 2;
  StateT<R> S;
  CoefT<R> c;
  R* scratch;

  __host__ __device__ void bind(const StateT<R>& s, const CoefT<R>& cc) {
    S = s;
    c = cc;
  }
  __device__ int lines() const { return DIR == 0 ? S.M - 3 : S.N - 3; }
  __device__ int cells_per_line() const { return DIR == 0 ? S.N - 1 : S.M - 1; }
  __device__ int unknowns_per_line() const { return cells_per_line(); }
  __device__ int at(int lp, int p) const { return DIR == 0 ? p * S.W + lp : lp * S.W + p; }
  __device__ const R* vel() const { return DIR == 0 ? S.tu : S.tv; }

  __device__ void load_segment(LineSeg& LS, int line, int s) const {
    const bool ok = line < lines();
    const int lp = line + 3;
    if (s == SEG) {
      LS.nseg = ok ? (DIR == 0 ? S.mocj[lp] : S.moci[lp]) : 0;
      return;
    }
    if (!ok) return;
    const int n = DIR == 0 ? S.mocj[lp] : S.moci[lp];
    if (s >= n) return;
    const int w = S.W;
    SegD& d = LS.s[s];
    int first, last;
    bool br1, br2;
    if (DIR == 0) {
      first = S.dauj[lp * SEG + s];
      last = S.cuoij[lp * SEG + s];
      br1 = (first > 2) || ((first == 2) && ((S.h[1 * w + lp] + S.h[1 * w + lp - 1]) * 0.5 == c.NANGDAY));
      br2 = (last < S.N) || ((last == S.N) && ((S.h[S.N * w + lp] + S.h[S.N * w + lp - 1]) * 0.5 == c.NANGDAY));
    } else {
      first = S.daui[lp * SEG + s];
      last = S.cuoii[lp * SEG + s];
      br1 = (first > 2) || ((first == 2) && ((S.h[lp * w + first - 1] + S.h[(lp - 1) * w + first - 1]) * 0.5 == c.NANGDAY));
      br2 = (last < S.M) || ((last == S.M) && ((S.h[lp * w + last] + S.h[(lp - 1) * w + last]) * 0.5 == c.NANGDAY));
    }
    d.first = first;
    d.last = last;
    d.off = first + 1;
    d.rend = last - 1;  // rend < off: no interior row, nothing solved
    d.br1 = br1;
    d.br2 = br2;
    d.ran = d.qfirst = d.last_kind = d.xq_first = d.xq_last = 0;
  }

  // Walks a chunk cell by cell; the rows come from k_fs_rows (one coalesced
  // per-cell pass ahead of the sweep), only the segment ends are set here.
  struct Walker {
    int lp, si, pos;
    bool in;
    __device__ void init(const FSGen& G, const LineSeg& LS, int line, int c0) {
      lp = line + 3;
      si = 0;
      in = false;
    }
    __device__ void cell(const FSGen& G, const LineSeg& LS, int cc) {
      pos = cc + 2;
      while (si < LS.nseg && LS.s[si].last < pos) ++si;
      in = si < LS.nseg && LS.s[si].off <= pos && pos <= LS.s[si].rend;
    }
    __device__ void row(const FSGen& G, const LineSeg& LS, int e, R& A, R& B, R& C,
                        R& D) const {
      if (!in) {
        A = 0; B = 1; C = 0; D = 0;
        return;
      }
      G.row_in(LS.s[si], lp, pos, A, B, C, D);
    }
  };

  // The row of cell pos of line position lp inside segment d: as k_fs_rows
  // wrote it, then the segment's end conditions.
  __device__ void row_in(const SegD& d, int lp, int pos, R& A, R& B, R& C, R& D) const {
    load_row(lp, pos, A, B, C, D);
    end_rows(d, lp, pos, A, B, C, D);
  }
  __device__ void load_row(int lp, int pos, R& A, R& B, R& C, R& D) const {
    const size_t n = (size_t)S.W * S.H;
    const R* q = S.pre + at(lp, pos);
    A = q[0];
    B = q[n];
    C = q[2 * n];
    D = q[3 * n];
  }
  __device__ void end_rows(const SegD& d, int lp, int pos, R& A, R& B, R& C, R& D) const {
    const R* v = vel();
    if (pos == d.first + 1) {
      // the velocity at the segment's first cell is the previous cell's
      if (d.br1 || v[at(lp, d.first)] == 0) B = B + A;
      else D = D - A * S.FS[at(lp, d.first)];
      A = 0;
    }
    if (pos == d.last - 1) {
      // '&&' in the i-sweep (sediment_transport.cpp:304), '||' in the j-sweep (:153)
      const bool zero = v[at(lp, d.last)] == 0;
      if (DIR == 0 ? (d.br2 && zero) : (d.br2 || zero)) B = B + C;
      else D = D - C * S.FS[at(lp, d.last)];
      C = 0;
    }
  }

  // The rows of a line again, unknown by unknown in decreasing order (the
  // refinement's residuals): the same values the Walker gave pass A.
  struct RowCursor {
    int lp, si;
    __device__ void init(const FSGen& G, const LineSeg& LS, int line) {
      lp = line + 3;
      si = LS.nseg - 1;
    }
    __device__ void row(const FSGen& G, const LineSeg& LS, int q, R& A, R& B, R& C, R& D) {
      const int pos = q + 2;
      while (si >= 0 && LS.s[si].first > pos) --si;
      if (si < 0 || pos < LS.s[si].off || pos > LS.s[si].rend) {
        A = 0; B = 1; C = 0; D = 0;
        return;
      }
      G.row_in(LS.s[si], lp, pos, A, B, C, D);
    }
  };

  // FWD: the unknowns come in increasing order (init_fwd), else decreasing.
  struct Emitter {
    int lp, si;
    __device__ void init(const FSGen& G, const LineSeg& LS, int line) {
      lp = line + 3;
      si = LS.nseg - 1;
    }
    __device__ void init_fwd(const FSGen& G, const LineSeg& LS, int line) {
      lp = line + 3;
      si = -1;
    }
    template <bool FWD = false>
    __device__ void emit(const FSGen& G, const LineSeg& LS, double* xlast, int q, double x) {
      const int pos = q + 2;
      if constexpr (FWD) {
        while (si + 1 < LS.nseg && LS.s[si + 1].first <= pos) ++si;
      } else {
        while (si >= 0 && LS.s[si].first > pos) --si;
      }
      if (si < 0) return;
      const SegD& d = LS.s[si];
      if (pos < d.off || pos > d.rend) return;
      G.S.tFS[G.at(lp, pos)] = (x < 0) ? G.c.NDnen : x;
    }
  };

  __device__ void fixup(const LineSeg& LS, const double* xlast, int line, int s) const {
    const SegD& d = LS.s[s];
    if (d.rend < d.off) return;
    const int lp = line + 3;
    const R* v = vel();
    R* tFS = S.tFS;
    tFS[at(lp, d.first)] = (d.br1 || v[at(lp, d.first)] == 0) ? tFS[at(lp, d.first + 1)]
                                                               : S.FS[at(lp, d.first)];
    tFS[at(lp, d.last)] = (d.br2 || v[at(lp, d.last)] == 0) ? tFS[at(lp, d.last - 1)]
                                                             : S.FS[at(lp, d.last)];
  }
};

template <class R>
int launch_fs_sweep(const StateT<R>& S, const CoefT<R>& c, int dir, cudaStream_t st,
                    const Batch<R>& b) {
  const int ncells = dir == 0 ? S.N - 1 : S.M - 1;
  const int lines = dir == 0 ? S.M - 3 : S.N - 3;
  if (lines <= 0) return 0;
  const int P = line_chunks(ncells, 4);
  const int slots = sweep_slots(S, ncells, P);
  if (dir == 0) {
    if (S.refine) return launch_lines(FSGen<0, R, true>{S, c, S.lscratch}, P, lines, slots, st, b);
    return launch_lines(FSGen<0, R, false>{S, c, S.lscratch}, P, lines, slots, st, b);
  }
  if (S.refine) return launch_lines(FSGen<1, R, true>{S, c, S.lscratch}, P, lines, slots, st, b);
  return launch_lines(FSGen<1, R, false>{S, c, S.lscratch}, P, lines, slots, st, b);
}

template <class R>
int launch_sweep(const StateT<R>& S, const CoefT<R>& c, int dir, cudaStream_t st,
                 const Batch<R>& b) {
  const int ncells = dir == 0 ? S.N - 1 : S.M - 1;
  const int P = line_chunks(ncells, 4);
  if (S.refine) {
    if (dir == 0) return launch_dir<0, R, true>(S, c, st, P, b);
    return launch_dir<1, R, true>(S, c, st, P, b);
  }
  if (dir == 0) return launch_dir<0, R, false>(S, c, st, P, b);
  return launch_dir<1, R, false>(S, c, st, P, b);
}

template int launch_sweep<double>(const StateT<double>&, const CoefT<double>&, int, cudaStream_t,
                                  const Batch<double>&);
template int launch_sweep<float>(const StateT<float>&, const CoefT<float>&, int, cudaStream_t,
                                 const Batch<float>&);
template int launch_fs_sweep<double>(const StateT<double>&, const CoefT<double>&, int, cudaStream_t,
                                     const Batch<double>&);
template int launch_fs_sweep<float>(const StateT<float>&, const CoefT<float>&, int, cudaStream_t,
                                    const Batch<float>&);

}  // namespace hyd
