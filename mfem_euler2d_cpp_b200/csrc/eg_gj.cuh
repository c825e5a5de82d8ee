// Gauss-Jordan building blocks shared by the HDG condensation (eg_hdg.cu)
// and the DG block-Jacobi inverses (eg_dginv.cu): the FP64 tensor-core MMA,
// the pivot reciprocal and the warp-level pivot selection of a 4-column
// panel. Not part of the public C-ABI.
#pragma once
#include "eg_device.cuh"

namespace eg {

// ------------------------------------------- tensor-core Gauss-Jordan
// D = C + A B on the FP64 tensor pipe: m8n8k4, A row-major 8x4 (one element
// per lane: row lane/4, column lane%4), B column-major 4x8 (row lane%4,
// column lane/4), C/D 8x8 (two elements per lane: row lane/4, columns
// 2*(lane%4) and 2*(lane%4)+1).
__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Reciprocal of a pivot: hardware estimate refined by two Newton-Raphson
// steps r <- r + r (1 - x r) (quadratic convergence from the ~2^-20 estimate;
// result within one unit in the last place of 1/x). The estimate flushes
// subnormal inputs and results to zero, so magnitudes outside
// [2^-1020, 2^1020] (and zero, infinities, NaN) take IEEE division instead.
__device__ __forceinline__ double pivot_reciprocal(double x) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-1020 && ax <= 0x1p+1020)) return 1.0 / x;
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}


// One warp chooses the 4 pivots of a panel staged in `pan` (rows x 4 panel
// columns) by partial pivoting over the rows not yet used: largest magnitude
// of the column after eliminating the panel's earlier pivots, first row on
// ties, NaN never chosen (MFEM LUFactors::Factor). It then publishes T^{-1}
// of the pivot block (row-major 4x4 in `fac`), the pivot rows (`pivs`) and
// their unknown indices (`invp`), and turns the pivot rows of the staged A
// operand into T_r - e_r. Returns false for a zero pivot (singular cell).
//
// The search is a dependent chain, so it is kept short: magnitudes are
// compared as IEEE bit patterns (integer compares, warp max/min reductions),
// and the column searched at step j+1 is formed fraction-free from the
// exact values of step j, p (w_{j+1} - (w_j / p) pw_{j+1}) = p w_{j+1} -
// w_j pw_{j+1}, whose magnitudes order the rows as the eliminated column
// does (common factor |p|). The exact elimination with multipliers
// w_j * (1/p), which yields the pivot rows and the multipliers of T's LU
// factors, runs beside the search instead of in front of it.
// With prow_all set, prow_all[jbase + c] also receives the pivot row of
// panel column c (the row permutation an explicit inverse needs).
template <int M, int KR>
__device__ __forceinline__ bool gj_select_pivots(int jbase, double (*pan)[4], double *fac, int *pivs,
                                                 unsigned char *used, int *invp, int lane,
                                                 int *prow_all = nullptr) {
  constexpr unsigned long long kAbs = 0x7fffffffffffffffull, kInf = 0x7ff0000000000000ull;
  constexpr int kNone = 0x7fffffff;
  double w[KR][4], key[KR], lm[KR][3];
  bool un[KR];
#pragma unroll
  for (int k = 0; k < KR; ++k) {
    const int i = lane + 32 * k;
    un[k] = i < M && !used[i];
#pragma unroll
    for (int c = 0; c < 4; ++c) w[k][c] = un[k] ? pan[i][c] : 0.;
    key[k] = w[k][0];
#pragma unroll
    for (int c = 0; c < 3; ++c) lm[k][c] = 0.;
  }
  int prow[4];
  double U[4][4], dinv[4], L[4][4];
#pragma unroll
  for (int jj = 0; jj < 4; ++jj) {
    unsigned long long best = 0ull;
    int idx = kNone;
#pragma unroll
    for (int k = 0; k < KR; ++k) {
      const unsigned long long bits = (unsigned long long)__double_as_longlong(key[k]) & kAbs;
      if (un[k] && bits <= kInf && (idx == kNone || bits > best)) {
        best = bits;
        idx = lane + 32 * k;
      }
    }
    const unsigned hi = (unsigned)(best >> 32), lo = (unsigned)best;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const bool c1 = idx != kNone && hi == mhi;
    const unsigned mlo = __reduce_max_sync(0xffffffffu, c1 ? lo : 0u);
    const bool c2 = c1 && lo == mlo;
    const int bi = (int)__reduce_min_sync(0xffffffffu, c2 ? (unsigned)idx : (unsigned)kNone);
    if ((mhi == 0u && mlo == 0u) || bi >= M) return false;
    prow[jj] = bi;
    const int owner = bi & 31, kk = bi >> 5;
    // the pivot row (eliminated by pivots 0..jj-1) and its multipliers
    double pw[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double v = 0.;
#pragma unroll
      for (int k = 0; k < KR; ++k)
        if (k == kk) v = w[k][c];
      pw[c] = c >= jj ? __shfl_sync(0xffffffffu, v, owner) : 0.;
    }
#pragma unroll
    for (int cc = 0; cc < jj; ++cc) {
      double v = 0.;
#pragma unroll
      for (int k = 0; k < KR; ++k)
        if (k == kk) v = lm[k][cc];
      L[jj][cc] = __shfl_sync(0xffffffffu, v, owner);
    }
#pragma unroll
    for (int k = 0; k < KR; ++k)
      if (k == kk && lane == owner) un[k] = false;
#pragma unroll
    for (int c = 0; c < 4; ++c) U[jj][c] = pw[c];
    const double inv = pivot_reciprocal(pw[jj]);
    dinv[jj] = inv;
    if (jj < 3) {
      // the column searched next, fraction-free (no reciprocal on the chain)
#pragma unroll
      for (int k = 0; k < KR; ++k) key[k] = fma(pw[jj], w[k][jj + 1], -(w[k][jj] * pw[jj + 1]));
      // exact elimination of the remaining panel columns
#pragma unroll
      for (int k = 0; k < KR; ++k) {
        const double l = w[k][jj] * inv;
        lm[k][jj] = l;
#pragma unroll
        for (int c = jj + 1; c < 4; ++c) w[k][c] -= l * pw[c];
      }
    }
  }
  // T^{-1}: lane c < 4 solves T x = e_c with the factors (L, U, 1/pivots)
  if (lane < 4) {
    double y[4];
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) {
      double v = rr == lane ? 1. : 0.;
#pragma unroll
      for (int cc = 0; cc < rr; ++cc) v -= L[rr][cc] * y[cc];
      y[rr] = v;
    }
#pragma unroll
    for (int rr = 3; rr >= 0; --rr) {
      double v = y[rr];
#pragma unroll
      for (int cc = rr + 1; cc < 4; ++cc) v -= U[rr][cc] * y[cc];
      y[rr] = v * dinv[rr];
    }
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) fac[rr * 4 + lane] = y[rr];
    const int pr = lane == 0 ? prow[0] : lane == 1 ? prow[1] : lane == 2 ? prow[2] : prow[3];
    pivs[lane] = pr;
    used[pr] = 1;
    invp[pr] = jbase + lane;
    if (prow_all) prow_all[jbase + lane] = pr;
    pan[pr][lane] -= 1.;  // A operand T_r - e_r
  }
  return true;
}


// ------------------------------------ two-phase Gauss-Jordan (A in smem)
// One warp chooses the 4 pivots of the panel whose columns are Acol[c*LDA+i]
// (c < 4, column-major, rows i < M) among the rows not yet used, by row
// partial pivoting: the row of largest magnitude in the column after the
// panel's earlier pivots are eliminated (MFEM LUFactors::Factor). The search
// runs fraction-free: the column searched at step s is p w - w_s pw over the
// previous step's values (scaled by the earlier pivots, which orders the rows
// as the eliminated column does), so no reciprocal sits on the chain. One
// warp max-reduction per step on a packed key (the top magnitude bits of the
// IEEE pattern and RMAX - row, so ties go to the first row; with 7 row bits
// (M <= 128) magnitudes within 2^-13 of each other count as ties, with 8 bits
// (M <= 256) within 2^-12, a choice as stable as the exact one);
// the pivot row reaches every lane through shared memory (rowbuf). Writes the
// pivot rows (pivs), marks them used and records their unknown index (invp);
// returns false for a zero column (singular cell; the remaining pivots are
// the first unused rows, so the caller's loop stays well defined).
template <int M, int KR, int LDA>
__device__ __forceinline__ bool gj_pick_pivots(int jbase, const double *Acol, double (*rowbuf)[4], int *pivs,
                                               unsigned char *used, int *invp, int lane) {
  static_assert(M <= 256, "pivot key holds at most 8 row bits");
  constexpr int RB = M <= 128 ? 7 : 8;
  constexpr unsigned RMAX = (1u << RB) - 1u;
  double w[KR][4];
  bool un[KR];
#pragma unroll
  for (int k = 0; k < KR; ++k) {
    const int i = lane + 32 * k;
    un[k] = i < M && !used[i];
#pragma unroll
    for (int c = 0; c < 4; ++c) w[k][c] = un[k] ? Acol[c * LDA + i] : 0.;
  }
  int prow[4];
  bool ok = true;
#pragma unroll
  for (int jj = 0; jj < 4; ++jj) {
    unsigned best = 0u;
#pragma unroll
    for (int k = 0; k < KR; ++k) {
      const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(w[k][jj]) >> 32) & 0x7fffffffu;
      const unsigned pk =
          (un[k] && hi <= 0x7ff00000u) ? (((hi >> RB) << RB) | (RMAX - (unsigned)(lane + 32 * k))) : 0u;
      best = pk > best ? pk : best;
    }
    const unsigned mb = __reduce_max_sync(0xffffffffu, best);
    int bi = (int)(RMAX - (mb & RMAX));
    if ((mb >> RB) == 0u) {
      ok = false;
      int cand = 0x7fffffff;
#pragma unroll
      for (int k = KR - 1; k >= 0; --k)
        if (un[k]) cand = lane + 32 * k;
      bi = (int)__reduce_min_sync(0xffffffffu, (unsigned)cand);
    }
    prow[jj] = bi;
    if (jj < 3) {
      __syncwarp();
      double pw[4];
#pragma unroll
      for (int c = jj; c < 4; ++c) pw[c] = jj == 0 ? Acol[c * LDA + bi] : rowbuf[bi][c];
#pragma unroll
      for (int k = 0; k < KR; ++k) {
        const int i = lane + 32 * k;
        if (i == bi) un[k] = false;
#pragma unroll
        for (int c = jj + 1; c < 4; ++c) w[k][c] = fma(pw[jj], w[k][c], -(w[k][jj] * pw[c]));
        if (un[k]) {
#pragma unroll
          for (int c = jj + 1; c < 4; ++c) rowbuf[i][c] = w[k][c];
        }
      }
    }
  }
  if (lane < 4) {
    const int pr = lane == 0 ? prow[0] : lane == 1 ? prow[1] : lane == 2 ? prow[2] : prow[3];
    pivs[lane] = pr;
    used[pr] = 1;
    invp[pr] = jbase + lane;
  }
  return ok;
}

// T^{-1} (row-major 4x4 in fac) of the pivot block T[r][c] = Acol[c*LDA +
// pivs[r]], by lanes 0..3 of one warp: LU of T in pivot order (no further
// pivoting: the rows were chosen by partial pivoting), then lane c solves
// T x = e_c. Afterwards the pivot rows of the panel hold T_r - e_r, the A
// operand that turns the update of a pivot row into its normalisation.
template <int LDA>
__device__ __forceinline__ void gj_pivot_block_inverse(double *Acol, const int *pivs, double *fac, int lane) {
  if (lane < 4) {
    double T[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) T[r][c] = Acol[c * LDA + pivs[r]];
    double dinv[4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      dinv[kk] = pivot_reciprocal(T[kk][kk]);
#pragma unroll
      for (int r = kk + 1; r < 4; ++r) {
        const double l = T[r][kk] * dinv[kk];
        T[r][kk] = l;
#pragma unroll
        for (int c = kk + 1; c < 4; ++c) T[r][c] = fma(-l, T[kk][c], T[r][c]);
      }
    }
    double y[4];
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) {
      double v = rr == lane ? 1. : 0.;
#pragma unroll
      for (int cc = 0; cc < rr; ++cc) v = fma(-T[rr][cc], y[cc], v);
      y[rr] = v;
    }
#pragma unroll
    for (int rr = 3; rr >= 0; --rr) {
      double v = y[rr];
#pragma unroll
      for (int cc = 3; cc > rr; --cc) v = fma(-T[rr][cc], y[cc], v);
      y[rr] = v * dinv[rr];
    }
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) fac[rr * 4 + lane] = y[rr];
  }
  __syncwarp();
  if (lane < 4) Acol[lane * LDA + pivs[lane]] -= 1.;
}

// Shapes of the two-phase Gauss-Jordan for an M x M cell matrix and NR
// right-hand sides (WR x WC warps over 8x8 tiles: 2 x 4 when two or three
// CTAs share an SM, 4 x 4 when one CTA fills it).
template <int M_, int NR_, int WR_ = 2, int WC_ = 4>
struct Gj2Cfg {
  static constexpr int M = M_, NR = NR_;
  static constexpr int MT = (M + 7) / 8;  // 8x8 tiles per side of A
  // stride of A: LDA % 8 in {2, 6} makes a warp's tile loads conflict-free
  static constexpr int LDA = ((M + 2) % 8 == 6 || (M + 2) % 8 == 2) ? M + 2 : ((M + 6) / 8) * 8 + 6;
  static constexpr int NRT = (NR + 7) / 8;
  static constexpr int WR = WR_, WC = WC_, THREADS = 32 * WR * WC;
  static constexpr int TRW = (MT + WR - 1) / WR;   // row tiles per warp
  static constexpr int TCA = (MT + WC - 1) / WC;   // A column tiles per warp
  static constexpr int TCW = (NRT + WC - 1) / WC;  // right-hand-side column tiles per warp
  static constexpr int NPAN = M / 4;
  static constexpr int KR = (M + 31) / 32;
  static constexpr int NP = 8 * MT, NQ = 8 * TCW * WC;
  // A, later reused for the outputs (M x NR at stride M + 1)
  static constexpr size_t DYN =
      sizeof(double) * (size_t)(LDA * M > (M + 1) * NR ? LDA * M : (M + 1) * NR);
};

// Phase 1 of the two-phase Gauss-Jordan (C: a Gj2Cfg): reduce the cell
// matrix A (shared memory, column-major, stride C::LDA) in 4-column panels
// with row partial pivoting. Warp 0 picks each panel's pivots and forms
// T^{-1}; the other warps copy the pivot rows' trailing columns; then every
// warp updates its trailing 8x8 tiles with one m8n8k4 FP64 MMA each
// (W_i -= a_i T^{-1} W_top, a_i = T_r - e_r on pivot rows), loads first,
// then MMAs, then stores. The panel columns are never written again:
// together with fac (T^{-1}) and pivs they record the elimination.
// The caller's `side(p, t, nt)` runs on the other warps (thread t of nt)
// while warp 0 searches panel p's pivots: work that does not touch A (the
// condensation stages its right-hand sides there), which fills the time
// those warps would spend waiting at the barrier.
struct Gj2NoSide {
  __device__ void operator()(int, int, int) const {}
};
template <class C, class Side = Gj2NoSide>
__device__ __forceinline__ void gj2_reduce(double *A, double (*topA)[C::NP], double (*rowbuf)[4], double (*fac)[16],
                                           int (*pivs)[4], unsigned char *used, int *invp, int *sing,
                                           const Side &side = Side()) {
  constexpr int M = C::M, LDA = C::LDA, WR = C::WR, WC = C::WC, TRW = C::TRW, TCA = C::TCA;
  constexpr int NPAN = C::NPAN, KR = C::KR, NP = C::NP, MT = C::MT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = warp % WR, wc = warp / WR;
  const int gq = lane >> 2, tq = lane & 3;
#pragma unroll 1
    for (int p = 0; p < NPAN; ++p) {
      const int j = 4 * p;
      double *Acol = A + (size_t)j * LDA;
      if (warp == 0) {
        if (!gj_pick_pivots<M, KR, LDA>(j, Acol, rowbuf, pivs[p], used, invp, lane) && lane == 0) *sing = 1;
      } else {
        side(p, threadIdx.x - 32, C::THREADS - 32);
      }
      __syncthreads();
      if (warp == 0) {
        gj_pivot_block_inverse<LDA>(Acol, pivs[p], fac[p], lane);
      } else {
        // the pivot rows' trailing columns (zero left of column j + 4)
        for (int t = threadIdx.x - 32; t < 4 * NP; t += C::THREADS - 32) {
          const int rr = t / NP, col = t % NP;
          topA[rr][col] = (col >= j + 4 && col < M) ? A[pivs[p][rr] + (size_t)col * LDA] : 0.;
        }
      }
      __syncthreads();
      const int tstart = (j + 4) >> 3;
      if (tstart < MT) {
        const double *F = fac[p];
        const double f0 = F[4 * tq], f1 = F[4 * tq + 1], f2 = F[4 * tq + 2], f3 = F[4 * tq + 3];
        double af[TRW];
#pragma unroll
        for (int a = 0; a < TRW; ++a) {
          const int row = (wr + a * WR) * 8 + gq;
          af[a] = row < M ? -Acol[tq * LDA + row] : 0.;
        }
#pragma unroll
        for (int b = 0; b < TCA; ++b) {
          const int tj = wc + b * WC;
          if (tj >= tstart && tj < MT) {
            const int colb = tj * 8 + gq;
            const double bf = f0 * topA[0][colb] + f1 * topA[1][colb] + f2 * topA[2][colb] + f3 * topA[3][colb];
            const int col = tj * 8 + 2 * tq;
            double d[TRW][2];
#pragma unroll
            for (int a = 0; a < TRW; ++a) {
              const int row = (wr + a * WR) * 8 + gq;
              d[a][0] = (row < M && col < M) ? A[row + (size_t)col * LDA] : 0.;
              d[a][1] = (row < M && col + 1 < M) ? A[row + (size_t)(col + 1) * LDA] : 0.;
            }
#pragma unroll
            for (int a = 0; a < TRW; ++a) dmma_m8n8k4(d[a][0], d[a][1], af[a], bf);
#pragma unroll
            for (int a = 0; a < TRW; ++a) {
              const int row = (wr + a * WR) * 8 + gq;
              if (row < M && col >= j + 4 && col < M) A[row + (size_t)col * LDA] = d[a][0];
              if (row < M && col + 1 >= j + 4 && col + 1 < M) A[row + (size_t)(col + 1) * LDA] = d[a][1];
            }
          }
        }
      }
      __syncthreads();
    }
}

// Phase 2: replay the recorded panels on right-hand sides held in registers
// as the warp's 8x8 tiles (rows (wr + a WR) 8 + gq, columns (wc + b WC) 8 +
// 2 tq + h): per panel the pivot rows are published (topR, double-buffered)
// and one MMA per tile applies the panel's update. Leaves the rows in pivot
// order: row w holds unknown invp[w].
template <class C, int TCW>
__device__ __forceinline__ void gj2_replay(const double *A, const double (*fac)[16], const int (*pivs)[4],
                                           double (*topR)[4][8 * TCW * C::WC], double (&acc)[C::TRW][TCW][2]) {
  constexpr int M = C::M, LDA = C::LDA, WR = C::WR, WC = C::WC, TRW = C::TRW, NPAN = C::NPAN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = warp % WR, wc = warp / WR;
  const int gq = lane >> 2, tq = lane & 3;
#pragma unroll 1
    for (int p = 0; p < NPAN; ++p) {
      const int j = 4 * p, pb = p & 1;
      const int pr0 = pivs[p][0], pr1 = pivs[p][1], pr2 = pivs[p][2], pr3 = pivs[p][3];
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int rbase = (wr + a * WR) * 8;
        // warp-uniform: does this tile row hold one of the pivot rows?
        if (!((unsigned)(pr0 - rbase) < 8u || (unsigned)(pr1 - rbase) < 8u || (unsigned)(pr2 - rbase) < 8u ||
              (unsigned)(pr3 - rbase) < 8u))
          continue;
        const int row = rbase + gq;
        const int rr = row == pr0 ? 0 : row == pr1 ? 1 : row == pr2 ? 2 : row == pr3 ? 3 : -1;
        if (rr >= 0) {
#pragma unroll
          for (int b = 0; b < TCW; ++b) {
            const int col = (wc + b * WC) * 8 + 2 * tq;
            topR[pb][rr][col] = acc[a][b][0];
            topR[pb][rr][col + 1] = acc[a][b][1];
          }
        }
      }
      __syncthreads();
      const double *Acol = A + (size_t)j * LDA;
      const double *F = fac[p];
      const double f0 = F[4 * tq], f1 = F[4 * tq + 1], f2 = F[4 * tq + 2], f3 = F[4 * tq + 3];
      double af[TRW];
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int row = (wr + a * WR) * 8 + gq;
        af[a] = row < M ? -Acol[tq * LDA + row] : 0.;
      }
#pragma unroll
      for (int b = 0; b < TCW; ++b) {
        const int colb = (wc + b * WC) * 8 + gq;
        const double bf = f0 * topR[pb][0][colb] + f1 * topR[pb][1][colb] + f2 * topR[pb][2][colb] +
                          f3 * topR[pb][3][colb];
#pragma unroll
        for (int a = 0; a < TRW; ++a) dmma_m8n8k4(acc[a][b][0], acc[a][b][1], af[a], bf);
      }
    }
}

}  // namespace eg
