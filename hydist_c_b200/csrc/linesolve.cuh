// linesolve.cuh -- partitioned tridiagonal line solver for the ADI sweeps.
//
// One CTA solves L adjacent lines at a time (LPB = 4; XPB = 8 for the
// 128-chunk column sweeps; a persistent loop walks the line groups). Each
// line is split into P chunks of consecutive cells; thread (chunk k, line l)
// = threadIdx.x = k*L + l, so with L = 4 a warp covers 8 chunks x 4 adjacent
// lines and every global access of a column sweep reads 4 adjacent columns
// (one 32-byte sector), with L = 8 4 chunks x 8 columns (64 bytes).
//
// The line's tridiagonal system (all wet segments of the line, identity rows
// between them) is solved by the partition method:
//   pass A  each chunk eliminates its interior rows forward, keeping the
//           spike of the unknown left of the chunk: x_r = y'_r + v'_r x_L
//           - c'_r x_{r+1}; (c', y', v') go to an L2-resident scratch slot;
//           the chunk's last unknown is a separator. The first interior
//           row in terms of both neighbouring separators is accumulated on
//           the way (x_0 = sum_k P_k (y'_k + v'_k x_L) + P_L x_R with
//           P_{k+1} = -c'_k P_k), the last one is the final state;
//   reduce  the separators form a tridiagonal Schur-complement system of P
//           unknowns per line, solved by parallel cyclic reduction in
//           shared memory;
//   pass C  backward substitution of every interior unknown, emitted to
//           the mesh fields as it is produced; then the per-segment end
//           fix-ups run.
// The row coefficients are generated on the fly by a generator class (the
// reference builds them in global arrays a1..d2, AA..DD first,
// UVZSolver_multithread.cpp:210-470, and solves each segment serially with
// tridiag(), :19-43).
#pragma once

#include "common.cuh"

namespace hyd {

constexpr int LPB = 4;  // lines per CTA
constexpr int XPB = 8;  // lines per CTA of the 128-chunk column sweeps

// One wet segment of a line, with its system layout.
struct SegD {
  int first, last;
  int off, rend;  // absolute rows [off, rend] of the segment's system
  unsigned char br1, br2, ran, qfirst, last_kind, xq_first, xq_last, pad;
};

struct LineSeg {
  int nseg;
  SegD s[SEG];
};

// Shared-memory layout of one CTA (R: the generator's arithmetic type).
template <class R, int P, int L = LPB>
struct LSShared {
  LineSeg seg[L];
  R sep[4][P * L];   // separator rows a, b, c, d
  R tri[6][P * L];   // yF vF wF yL vL wL per chunk
  R red[4][P * L];   // reduced system during PCR
  R xsep[P * L];     // separator solutions
  double xlast[L][SEG];  // solution at each segment's last row
};

// A plain division: with FP64 it keeps the rounding of the reference's
// formulas within one ulp.
template <class R>
__device__ __forceinline__ R rcp(R x) { return R(1) / x; }

// PCR levels for P separators per line
constexpr int pcr_levels(int P) { return P <= 1 ? 0 : 1 + pcr_levels(P / 2); }

// dynamic shared memory of one CTA: LSShared, and with refinement the PCR
// multipliers
template <class R, int P, int L = LPB>
constexpr size_t line_smem(bool refine) {
  return sizeof(LSShared<R, P, L>) + (refine ? (size_t)2 * pcr_levels(P) * P * L * sizeof(R) : 0);
}

// Gen::MIN_BLOCKS: resident CTAs per SM the P = 128 solver is compiled for
// (2 caps registers at 64 per thread). The solvers for shorter lines (fewer
// chunks, smaller CTAs) are compiled for at least 512 threads per SM, the
// row sweeps' for as many as their P = 128 solver (at most 32 CTAs): left
// uncapped, the row sweeps' short-line solvers took up to 198 registers and
// ran 8 warps per SM; the column sweeps' spill under the 64-register cap.
template <class Gen, int P, int L>
constexpr int line_min_blocks() {
  constexpr int k = (L * P >= 512) ? 1 : 512 / (L * P);
  constexpr int b = Gen::DIRECTION == 1 ? k * Gen::MIN_BLOCKS : k;
  if (L * P >= 1024) return 1;  // one CTA per SM, 64 registers per thread
  return (P == 128 && L == LPB) ? Gen::MIN_BLOCKS : (b > 32 ? 32 : b);
}

// The launch solves line groups 0 .. ngroups-1 of L lines from line0 on.
// BATCH: the groups of every member of a batch, gpm groups per member (the
// member of group g is g / gpm, its state and coefficients bound into a
// copy of G0 for that group); the persistent grid walks them all, each CTA
// with its own scratch slot of G0's scratch.
template <class Gen, int P, int L = LPB, int BATCH = 0>
__global__ void __launch_bounds__(L * P, line_min_blocks<Gen, P, L>())
    k_line_solve(Gen G0, int line0, int ngroups, Batch<typename Gen::Real> bt, int gpm) {
  using R = typename Gen::Real;
  // sizes and scratch from G0: the same for every member of a batch
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LSShared<R, P, L>& sh = *reinterpret_cast<LSShared<R, P, L>*>(smem_raw);
  // with refinement: the PCR multipliers, 2 per level per thread
  constexpr int PL = P * L;
  R* pm = reinterpret_cast<R*>(smem_raw + sizeof(LSShared<R, P, L>));
  const int tid = threadIdx.x;
  const int l = tid % L, k = tid / L;
  const int cidx = k * L + l;
  const int U = G0.unknowns_per_line();
  // scratch slot of this CTA: c', y', v' per unknown, and with refinement
  // also the rows A, B, C, D (Gen::SCRATCH_ARRAYS arrays of U x L)
  const size_t UL = (size_t)U * L;
  R* scr = G0.scratch + (size_t)blockIdx.x * Gen::SCRATCH_ARRAYS * UL;
  R* sc_c = scr;
  R* sc_y = scr + UL;
  R* sc_v = scr + 2 * UL;
  const int ncells = G0.cells_per_line();
  const int upc = Gen::UPC;

  // one group of L lines: gg-th of its scenario, with that scenario's G
  auto solve_group = [&](const Gen& G, int gg) {
    const int line = line0 + gg * L + l;
    // ---- segment descriptors of the group's lines
    for (int e = tid; e < L * (SEG + 1); e += blockDim.x) {
      const int ll = e / (SEG + 1), s = e % (SEG + 1);
      G.load_segment(sh.seg[ll], line0 + gg * L + ll, s);
    }
    __syncthreads();
    const LineSeg& LS = sh.seg[l];
    // ---- chunk bounds (balanced split of the line's cells)
    const int c0 = (int)(((long long)k * ncells) / P);
    const int c1 = (int)(((long long)(k + 1) * ncells) / P);
    const int q0 = c0 * upc, nu = (c1 - c0) * upc;  // chunk unknowns [q0, q0+nu)

    // ---- pass A: forward elimination of the interior, separator row
    {
      typename Gen::Walker W;
      W.init(G, LS, line, c0);
      // (with no interior row, the unknown left of the separator is x_L)
      R cp = 0, yp = 0, vp = 1;
      // first interior row in terms of both separators, accumulated forward:
      // x_0 = sum_k P_k (y'_k + v'_k x_L) + P_L x_R, P_0 = 1, P_{k+1} = -c'_k P_k
      R Pk = 1, fy = 0, fv = 0;
      int s = 0;
      for (int c = c0; c < c1; ++c) {
        W.cell(G, LS, c);
#pragma unroll
        for (int e = 0; e < Gen::UPC; ++e, ++s) {
          R A, B, C, D;
          W.row(G, LS, e, A, B, C, D);
          if (s == nu - 1) {
            sh.sep[0][cidx] = A;
            sh.sep[1][cidx] = B;
            sh.sep[2][cidx] = C;
            sh.sep[3][cidx] = D;
          } else {
            R m;
            if (s == 0) {
              m = rcp(B);
              cp = C * m;
              yp = D * m;
              vp = -A * m;
            } else {
              m = rcp(B - A * cp);
              yp = (D - A * yp) * m;
              vp = -A * vp * m;
              cp = C * m;
            }
            const size_t o = (size_t)(q0 + s) * L + l;
            if constexpr (Gen::REFINE && !Gen::ROWS_AGAIN) {
              // the interior rows, for the residual
              scr[3 * UL + o] = A;
              scr[4 * UL + o] = B;
              scr[5 * UL + o] = C;
              scr[6 * UL + o] = D;
            }
            sc_c[o] = cp;
            sc_y[o] = yp;
            sc_v[o] = vp;
            fy += Pk * yp;
            fv += Pk * vp;
            Pk *= -cp;
          }
        }
      }
      // first and last interior rows in terms of the neighbouring separators
      sh.tri[0][cidx] = fy;
      sh.tri[1][cidx] = fv;
      sh.tri[2][cidx] = Pk;
      sh.tri[3][cidx] = yp;
      sh.tri[4][cidx] = vp;
      sh.tri[5][cidx] = -cp;
    }
    __syncthreads();
    // ---- reduced (Schur complement) system of the separators
    R ra, rb, rc, rd;
    {
      const R as = sh.sep[0][cidx], bs = sh.sep[1][cidx], cs = sh.sep[2][cidx],
              ds = sh.sep[3][cidx];
      const R yL = sh.tri[3][cidx], vL = sh.tri[4][cidx], wL = sh.tri[5][cidx];
      R yF = 0, vF = 0, wF = 0;
      if (k + 1 < P) {
        const int n1 = cidx + L;
        yF = sh.tri[0][n1];
        vF = sh.tri[1][n1];
        wF = sh.tri[2][n1];
      }
      ra = as * vL;
      rb = bs + as * wL + cs * vF;
      rc = cs * wF;
      rd = ds - as * yL - cs * yF;
    }
    // parallel cyclic reduction (the refinement keeps each level's
    // multipliers for its correction)
    for (int st = 1, lvl = 0; st < P; st <<= 1, ++lvl) {
      sh.red[0][cidx] = ra;
      sh.red[1][cidx] = rb;
      sh.red[2][cidx] = rc;
      sh.red[3][cidx] = rd;
      __syncthreads();
      R am = 0, bm = 1, cm = 0, dm = 0, an = 0, bn = 1, cn = 0, dn = 0;
      if (k - st >= 0) {
        const int o = cidx - st * L;
        am = sh.red[0][o];
        bm = sh.red[1][o];
        cm = sh.red[2][o];
        dm = sh.red[3][o];
      }
      if (k + st < P) {
        const int o = cidx + st * L;
        an = sh.red[0][o];
        bn = sh.red[1][o];
        cn = sh.red[2][o];
        dn = sh.red[3][o];
      }
      __syncthreads();
      const R k1 = ra / bm, k2 = rc / bn;
      if constexpr (Gen::REFINE) {
        pm[(2 * lvl) * PL + cidx] = k1;
        pm[(2 * lvl + 1) * PL + cidx] = k2;
      }
      const R na = -am * k1, nc = -cn * k2;
      const R nb = rb - cm * k1 - an * k2;
      const R nd = rd - dm * k1 - dn * k2;
      ra = na;
      rb = nb;
      rc = nc;
      rd = nd;
    }
    sh.xsep[cidx] = rd / rb;
    __syncthreads();
    // ---- pass C: back substitution and emission
    if constexpr (!Gen::REFINE) {
      const R xr = sh.xsep[cidx];
      const R xl = (k > 0) ? sh.xsep[cidx - L] : R(0);
      typename Gen::Emitter E;
      E.init(G, LS, line);
      E.emit(G, LS, sh.xlast[l], q0 + nu - 1, xr);
      R xn = xr;
#pragma unroll 4
      for (int t = nu - 2; t >= 0; --t) {
        const size_t o = (size_t)(q0 + t) * L + l;
        const R x = sc_y[o] + sc_v[o] * xl - sc_c[o] * xn;
        E.emit(G, LS, sh.xlast[l], q0 + t, x);
        xn = x;
      }
    } else {
      // one refinement pass. The back substitution stores x over y' and, as
      // soon as x_{t-1..t+1} are known, takes row t's residual
      // r = D - A x_{t-1} - B x_t - C x_{t+1} in FP64 from the stored rows
      // and eliminates the correction system A d = r backward through it:
      // d_t = h_t - a_t d_{t-1} - w_t d_R (d_R the chunk's separator), the
      // (a, h, w) over the rows' A, D, C. The separators' correction solves
      // the same Schur complement as pass A, so the reduction reuses pass
      // A's PCR multipliers; the chunk interiors are then substituted
      // forward and x + d is emitted in FP64.
      // Gen::ROWS_AGAIN: the rows are read again from where the generator
      // read them in pass A (the same values), not from the scratch, and
      // (a, h, w) go over the c', v' of the row they belong to (consumed by
      // then) and a fourth scratch array; else the stored rows' A, D, C.
      R* sA = Gen::ROWS_AGAIN ? sc_c : scr + 3 * UL;
      R* sB = scr + 4 * UL;
      R* sC = Gen::ROWS_AGAIN ? sc_v : scr + 5 * UL;
      R* sD = Gen::ROWS_AGAIN ? scr + 3 * UL : scr + 6 * UL;
      typename Gen::RowCursor cur;
      cur.init(G, LS, line);
      const R xr = sh.xsep[cidx];
      const R xl = (k > 0) ? sh.xsep[cidx - L] : R(0);
      R x_before_sep = 0;  // x of the chunk's last interior unknown
      R ha = 0, hy = 0, hw = -1;  // (a, h, w) of the row below the one eliminated
      R gy = 0, gw = 0, Q = 1;    // d of the last interior unknown: gy - gw d_R + Q d_L
      // row q (slot o), q decreasing from call to call
      auto eliminate = [&](size_t o, int q, R xm, R x, R xp) {
        R A, B, C, D;
        if constexpr (Gen::ROWS_AGAIN) {
          cur.row(G, LS, q, A, B, C, D);
        } else {
          A = sA[o];
          B = sB[o];
          C = sC[o];
          D = sD[o];
        }
        const R r = (R)((double)D - (double)A * (double)xm - (double)B * (double)x -
                        (double)C * (double)xp);
        const R m = rcp(B - C * ha);
        ha = A * m;
        hy = (r - C * hy) * m;
        hw = -C * hw * m;
        sA[o] = ha;
        sD[o] = hy;
        sC[o] = hw;
        gy += Q * hy;
        gw += Q * hw;
        Q *= -ha;
      };
      {
        R x1 = xr, x2 = 0;  // x_{t+1}, x_{t+2}
        for (int t = nu - 2; t >= 0; --t) {
          const size_t o = (size_t)(q0 + t) * L + l;
          const R x = sc_y[o] + sc_v[o] * xl - sc_c[o] * x1;
          sc_y[o] = x;
          if (t == nu - 2) x_before_sep = x;
          else eliminate(o + L, q0 + t + 1, x, x1, x2);
          x2 = x1;
          x1 = x;
        }
        // the first unknown: its left neighbour is the previous separator
        // (none at the line's start)
        if (nu >= 2) eliminate((size_t)q0 * L + l, q0, q0 > 0 ? xl : R(0), x1, x2);
      }
      // the first interior unknown's constant term, for the previous chunk
      sh.tri[0][cidx] = hy;
      __syncthreads();
      R rd2 = 0;
      if (nu >= 1) {
        // the separator row: its right neighbour is the next chunk's first
        // unknown (none at the line's end)
        const int q = q0 + nu - 1;
        const size_t o = (size_t)q * L + l;
        // the unknown left of the separator: the chunk's last interior one,
        // or the previous chunk's separator; right of it: the next chunk's
        // first unknown, its separator where that chunk holds nothing else
        const int nu_next = (k + 1 < P)
            ? ((int)(((long long)(k + 2) * ncells) / P) - c1) * upc : 0;
        const R xm = nu >= 2 ? x_before_sep : (q > 0 ? xl : R(0));
        const R xp = q + 1 < U ? (nu_next >= 2 ? sc_y[o + L] : sh.xsep[cidx + L]) : R(0);
        const R as = sh.sep[0][cidx], bs = sh.sep[1][cidx], cs = sh.sep[2][cidx],
                ds = sh.sep[3][cidx];
        const R rs = (R)((double)ds - (double)as * (double)xm - (double)bs * (double)xr -
                         (double)cs * (double)xp);
        const R hF = (k + 1 < P) ? sh.tri[0][cidx + L] : R(0);
        rd2 = rs - as * gy - cs * hF;
      }
      // the reduction with pass A's multipliers (one barrier per level: the
      // levels alternate between two buffers)
      {
        int lvl = 0;
        for (int st = 1; st < P; st <<= 1, ++lvl) {
          R* buf = sh.red[lvl & 1];
          buf[cidx] = rd2;
          __syncthreads();
          const R dm = (k - st >= 0) ? buf[cidx - st * L] : R(0);
          const R dn = (k + st < P) ? buf[cidx + st * L] : R(0);
          rd2 = rd2 - dm * pm[(2 * lvl) * PL + cidx] - dn * pm[(2 * lvl + 1) * PL + cidx];
        }
      }
      const R dr = rd2 / rb;
      sh.xsep[cidx] = dr;
      __syncthreads();
      {
        const R dl = (k > 0) ? sh.xsep[cidx - L] : R(0);
        typename Gen::Emitter E;
        E.init_fwd(G, LS, line);
        R dp = dl;
        for (int t = 0; t <= nu - 2; ++t) {
          const size_t o = (size_t)(q0 + t) * L + l;
          const R d = sD[o] - sA[o] * dp - sC[o] * dr;
          E.template emit<true>(G, LS, sh.xlast[l], q0 + t, (double)sc_y[o] + (double)d);
          dp = d;
        }
        if (nu >= 1) E.template emit<true>(G, LS, sh.xlast[l], q0 + nu - 1, (double)xr + (double)dr);
      }
    }
    __syncthreads();
    // ---- per-segment end fix-ups
    for (int e = tid; e < L * SEG; e += blockDim.x) {
      const int ll = e / SEG, s = e % SEG;
      if (s < sh.seg[ll].nseg) G.fixup(sh.seg[ll], sh.xlast[ll], line0 + gg * L + ll, s);
    }
    __syncthreads();
  };
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    if constexpr (BATCH != 0) {
      const int m = grp / gpm;
      Gen Gm = G0;
      Gm.bind(bt.S[m], bt.c[m]);
      solve_group(Gm, grp - m * gpm);
    } else {
      solve_group(G0, grp);
    }
  }
}

}  // namespace hyd
