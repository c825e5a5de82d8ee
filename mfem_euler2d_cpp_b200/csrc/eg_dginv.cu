// DG block Jacobi (PartialDGOperator::DiagonalBlocks, src/partial.cpp:265-298,
// factored as in src/linear.cpp:198-202 and applied by
// LinearSolver::Impl::Precondition, src/linear.cpp:66-75) without triangular
// sweeps. Both forms below pick the pivots LUFactors::Factor would choose
// (virtual row partial pivoting, eg_gj.cuh) and use the FP64 tensor cores.
//
// k <= 2 -- explicit inverses: each cell's m x m block is inverted in place
// by a register-resident Gauss-Jordan (the panel's columns, once eliminated,
// take the unit columns of the identity the inverse is built from: 2 m^3
// flops), written column-major and applied as a column-major block GEMV,
// one warp per cell, lanes over rows, 16-byte loads.
//
// k = 3..5 -- Gauss-Jordan records: phase 1 of the two-phase Gauss-Jordan
// (gj2_reduce: A in shared memory, 4-column panels, m^3 flops) and nothing
// more; the reduced block, the panels' T^{-1} and their pivot rows leave the
// SM as the record. The apply replays the elimination on the right-hand
// side, panel by panel, one warp per cell: it streams the m^2 doubles of the
// record once, the traffic of an explicit inverse, while the factor skips
// the 2 m^3 flops of replaying the elimination on the identity.
#include <algorithm>

#include "eg_cellmat.cuh"
#include "eg_gj.cuh"
#include "eg_bulk.cuh"
#include "eg_internal.h"

namespace eg {
namespace {

template <int Q, int WR, int WC>
struct GjInvCfg {
  static constexpr int P = Q * Q, M = 4 * P;
  static constexpr int MT = (M + 7) / 8;                       // 8x8 tiles per side
  static constexpr int TRW = (MT + WR - 1) / WR, TCW = (MT + WC - 1) / WC;
  static constexpr int MP = 8 * TRW * WR, NP = 8 * TCW * WC;  // padded to whole warp tile grids
  static constexpr int THREADS = 32 * WR * WC;
  static constexpr int LD = M + 1;          // odd staging stride: conflict-free columns
  static constexpr int KR = (M + 31) / 32;  // rows per lane in the pivot search
};

template <int Q, int WR, int WC, int MINB>
__global__ void __launch_bounds__(32 * WR *WC, MINB)
    dg_inverse_gj_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                         double *__restrict__ inv, int *err) {
  using C = GjInvCfg<Q, WR, WC>;
  constexpr int M = C::M, MP = C::MP, NP = C::NP, TRW = C::TRW, TCW = C::TCW, LD = C::LD, KR = C::KR;
  constexpr int NPAN = M / 4;
  __shared__ STab<Q> st;
  __shared__ double us[M], UT[16 * Q], FM[4 * Q * 16];
  __shared__ double pan[2][MP][4], top[2][4][NP];
  __shared__ double fac[2][16];  // T^{-1} of the panel's pivot block, row-major 4x4
  __shared__ int pivs[2][4];
  __shared__ int invp[MP], prow[M];
  __shared__ unsigned char used[MP];
  __shared__ int sing;
  extern __shared__ double dyn[];  // the block (column-major, stride LD), then its inverse (stride M)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = warp % WR, wc = warp / WR;
  const int gq = lane >> 2, tq = lane & 3;
  load_tables<Q>(st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += C::THREADS) us[i] = u[(size_t)e * M + i];
    __syncthreads();
    cell_traces<Q>(st, us, UT);
    __syncthreads();
    dg_face_matrices<Q>(UT, FM, g, fz, e);
    __syncthreads();
    build_cell_matrix<Q>(dyn, LD, st, us, FM, g);
    for (int i = threadIdx.x; i < MP; i += C::THREADS) {
      used[i] = i >= M ? 1 : 0;
      invp[i] = 0;
    }
    if (threadIdx.x == 0) sing = 0;
    __syncthreads();
    double acc[TRW][TCW][2];
#pragma unroll
    for (int a = 0; a < TRW; ++a) {
      const int row = (wr + a * WR) * 8 + gq;
#pragma unroll
      for (int b = 0; b < TCW; ++b) {
        const int col = (wc + b * WC) * 8 + 2 * tq;
        acc[a][b][0] = (row < M && col < M) ? dyn[row + (size_t)col * LD] : 0.;
        acc[a][b][1] = (row < M && col + 1 < M) ? dyn[row + (size_t)(col + 1) * LD] : 0.;
      }
    }
    // stage panel 0 (tile column 0, left half)
    if (wc == 0 && tq < 2) {
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int row = (wr + a * WR) * 8 + gq;
        pan[0][row][2 * tq] = acc[a][0][0];
        pan[0][row][2 * tq + 1] = acc[a][0][1];
      }
    }
    __syncthreads();
    if (warp == 0 && !gj_select_pivots<M, KR>(0, pan[0], fac[0], pivs[0], used, invp, lane, prow) && lane == 0)
      sing = 1;
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < NPAN && !sing; ++p) {
      const int j = 4 * p, pb = p & 1;
      const int pr0 = pivs[pb][0], pr1 = pivs[pb][1], pr2 = pivs[pb][2], pr3 = pivs[pb][3];
      const int tp = j >> 3, half = (j >> 2) & 1;
      // publish the pivot rows over every column; the panel's own columns
      // are replaced by the unit columns of the identity
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int row = (wr + a * WR) * 8 + gq;
        const int rr = row == pr0 ? 0 : row == pr1 ? 1 : row == pr2 ? 2 : row == pr3 ? 3 : -1;
        if (rr >= 0) {
#pragma unroll
          for (int b = 0; b < TCW; ++b) {
            const int col = (wc + b * WC) * 8 + 2 * tq;
            const bool in0 = col >= j && col < j + 4, in1 = col + 1 >= j && col + 1 < j + 4;
            top[pb][rr][col] = in0 ? (col - j == rr ? 1. : 0.) : acc[a][b][0];
            top[pb][rr][col + 1] = in1 ? (col + 1 - j == rr ? 1. : 0.) : acc[a][b][1];
          }
        }
      }
      // the same replacement in the accumulators: column j + c becomes
      // e_{pivot row of c}
      if ((tq >> 1) == half) {
        const int ra = (tq & 1) ? pr2 : pr0, rb = (tq & 1) ? pr3 : pr1;
#pragma unroll
        for (int b = 0; b < TCW; ++b) {
          if (wc + b * WC == tp) {
#pragma unroll
            for (int a = 0; a < TRW; ++a) {
              const int row = (wr + a * WR) * 8 + gq;
              acc[a][b][0] = row == ra ? 1. : 0.;
              acc[a][b][1] = row == rb ? 1. : 0.;
            }
          }
        }
      }
      __syncthreads();
      // A operands (row gq, column tq of each tile row): -W[row, panel], with
      // T_r - e_r on the pivot rows; B operands (row tq, column gq) = T^{-1} top
      double af[TRW];
#pragma unroll
      for (int a = 0; a < TRW; ++a) af[a] = -pan[pb][(wr + a * WR) * 8 + gq][tq];
      const double *F = fac[pb];
      const double f0 = F[4 * tq], f1 = F[4 * tq + 1], f2 = F[4 * tq + 2], f3 = F[4 * tq + 3];
      const bool more = p + 1 < NPAN;
      const int jn = j + 4, tstart = jn >> 3, nhalf = (jn >> 2) & 1, nb = pb ^ 1;
      const bool stager = more && wc == tstart % WC && (tq >> 1) == nhalf;
#pragma unroll
      for (int b = 0; b < TCW; ++b) {
        const int tj = wc + b * WC;
        if (tj * 8 < M) {  // tiles of padding columns stay zero
          const int col = tj * 8 + gq;
          const double bf = f0 * top[pb][0][col] + f1 * top[pb][1][col] + f2 * top[pb][2][col] +
                            f3 * top[pb][3][col];
#pragma unroll
          for (int a = 0; a < TRW; ++a) dmma_m8n8k4(acc[a][b][0], acc[a][b][1], af[a], bf);
          if (tj == tstart && stager) {
#pragma unroll
            for (int a = 0; a < TRW; ++a) {
              const int row = (wr + a * WR) * 8 + gq;
              pan[nb][row][2 * (tq & 1)] = acc[a][b][0];
              pan[nb][row][2 * (tq & 1) + 1] = acc[a][b][1];
            }
          }
        }
      }
      __syncthreads();
      if (more && warp == 0 && !gj_select_pivots<M, KR>(jn, pan[nb], fac[nb], pivs[nb], used, invp, lane, prow) &&
          lane == 0)
        sing = 1;
      __syncthreads();
    }
    if (sing) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_JACOBI);
      continue;
    }
    // W[w, slot] holds E[w, prow[slot]] of the reduced [A | I] = [P | P A^{-1}],
    // so A^{-1}[invp[w], prow[slot]] = W[w, slot]; stored column-major
#pragma unroll
    for (int a = 0; a < TRW; ++a) {
      const int row = (wr + a * WR) * 8 + gq;
      if (row < M) {
        const int i = invp[row];
#pragma unroll
        for (int b = 0; b < TCW; ++b) {
          const int col = (wc + b * WC) * 8 + 2 * tq;
          if (col < M) dyn[(size_t)prow[col] * M + i] = acc[a][b][0];
          if (col + 1 < M) dyn[(size_t)prow[col + 1] * M + i] = acc[a][b][1];
        }
      }
    }
    __syncthreads();
    double2 *dst = reinterpret_cast<double2 *>(inv + (size_t)e * M * M);
    const double2 *src = reinterpret_cast<const double2 *>(dyn);
    for (int i = threadIdx.x; i < M * M / 2; i += C::THREADS) dst[i] = src[i];
  }
}

// x_e = A_e^{-1} b_e, inverses column-major: one warp per cell, lane l holds
// rows 2l, 2l+1 (+ 64 s); the right-hand side is staged per warp in shared
// memory and broadcast column by column.
template <int M>
__global__ void __launch_bounds__(256) block_inverse_cm_apply_kernel(const double *__restrict__ inv, int nblocks,
                                                                     const double *__restrict__ b,
                                                                     double *__restrict__ x,
                                                                     const int *__restrict__ skip,
                                                                     const int *__restrict__ perm) {
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  constexpr int S = (M + 63) / 64;
  __shared__ double bs[8][M];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * 8 + warp;
  if (blk >= nblocks) return;  // warp-uniform; nothing below synchronises the CTA
  for (int i = lane; i < M; i += 32) bs[warp][i] = b[(size_t)blk * M + i];
  __syncwarp();
  const double *A = inv + (size_t)blk * M * M;
  double acc[S][2];
#pragma unroll
  for (int s = 0; s < S; ++s) acc[s][0] = acc[s][1] = 0.;
#pragma unroll 4
  for (int c = 0; c < M; ++c) {
    const double bc = bs[warp][c];
    const double2 *col = reinterpret_cast<const double2 *>(A + (size_t)c * M);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int r2 = lane + 32 * s;  // row pair
      if (2 * r2 < M) {
        const double2 v = __ldcs(col + r2);
        acc[s][0] = fma(v.x, bc, acc[s][0]);
        acc[s][1] = fma(v.y, bc, acc[s][1]);
      }
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int r2 = lane + 32 * s;
    if (2 * r2 < M) {
      if (perm == nullptr) {
        reinterpret_cast<double2 *>(x + (size_t)blk * M)[r2] = make_double2(acc[s][0], acc[s][1]);
      } else {  // row w of the stored inverse is row perm[w] of the true one
        const int *pb = perm + (size_t)blk * M;
        x[(size_t)blk * M + pb[2 * r2]] = acc[s][0];
        x[(size_t)blk * M + pb[2 * r2 + 1]] = acc[s][1];
      }
    }
  }
}

// ------------------------------------------------ Gauss-Jordan record (k = 3..5)
// Factor without the identity replay: phase 1 of the two-phase Gauss-Jordan
// (gj2_reduce) on the cell block, then its record leaves the SM as it is --
// the m x m reduced block column-major (the panel columns hold the
// eliminated entries, T_r - e_r on the pivot rows), T^{-1} of every panel
// (fac: NPAN x 16, row-major 4x4) and the panels' pivot rows (pivs) -- with
// the unknown order invp of the result rows (perm). The record holds as
// many bytes as an explicit inverse, so the apply streams the same traffic,
// but the factor does m^3 flops instead of the inverse's 3 m^3.
template <int Q, int MINB, int WR_ = 2, int WC_ = 4>
__global__ void __launch_bounds__(32 * WR_ *WC_, MINB)
    dg_gj_record_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                        double *__restrict__ rec, double *__restrict__ rec_fac, int *__restrict__ rec_pivs,
                        int *__restrict__ perm, int *err) {
  constexpr int M = 4 * Q * Q;
  using C = Gj2Cfg<M, M, WR_, WC_>;
  constexpr int NPAN = C::NPAN, KR = C::KR, NP = C::NP, LDA = C::LDA;
  __shared__ STab<Q> st;
  __shared__ double us[M], UT[16 * Q], FM[4 * Q * 16];
  __shared__ double topA[4][NP];
  __shared__ double rowbuf[KR * 32][4];
  __shared__ double fac[NPAN][16];
  __shared__ int pivs[NPAN][4];
  __shared__ int invp[KR * 32];
  __shared__ unsigned char used[KR * 32];
  __shared__ int sing;
  extern __shared__ __align__(16) double A[];
  load_tables<Q>(st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += C::THREADS) us[i] = u[(size_t)e * M + i];
    __syncthreads();
    cell_traces<Q>(st, us, UT);
    __syncthreads();
    dg_face_matrices<Q>(UT, FM, g, fz, e);
    __syncthreads();
    build_cell_matrix<Q>(A, LDA, st, us, FM, g);
    for (int i = threadIdx.x; i < KR * 32; i += C::THREADS) {
      used[i] = i >= M ? 1 : 0;
      invp[i] = 0;
    }
    if (threadIdx.x == 0) sing = 0;
    __syncthreads();
    // a panel's 4 columns (with T_r - e_r on its pivot rows) and its T^{-1}
    // are final once its update is done: the warps waiting while warp 0
    // searches panel p's pivots write out panel p - 1
    double *R = rec + (size_t)e * M * M;
    double *Fo = rec_fac + (size_t)e * NPAN * 16;
    const auto write_panel = [&](int q, int t, int nt) {
      for (int i = t; i < 4 * M; i += nt) R[(size_t)q * 4 * M + i] = A[(i % M) + (size_t)(4 * q + i / M) * LDA];
      for (int i = t; i < 16; i += nt) Fo[q * 16 + i] = fac[q][i];
    };
    const auto side = [&](int pp, int t, int nt) {
      if (pp > 0) write_panel(pp - 1, t, nt);
    };
    gj2_reduce<C>(A, topA, rowbuf, fac, pivs, used, invp, &sing, side);
    if (sing) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_JACOBI);
      continue;
    }
    write_panel(NPAN - 1, threadIdx.x, C::THREADS);
    for (int i = threadIdx.x; i < M; i += C::THREADS) {
      rec_pivs[(size_t)e * M + i] = pivs[i >> 2][i & 3];
      perm[(size_t)e * M + i] = invp[i];
    }
  }
}

// Shapes of the record apply: NB panel buffers per warp, W warps (cells) per
// CTA, sized so that two CTAs share an SM where they fit.
template <int M>
struct RecApplyCfg {
  static constexpr int NPAN = M / 4;
  static constexpr int NB = 3;                      // panels in flight per warp
  static constexpr int W = M <= 100 ? 8 : 4;        // warps (cells) per CTA
  static constexpr int PANEL = 4 * M;               // doubles per panel (contiguous in the record)
  static constexpr int PIVS = (M + 3) / 4 * 4;      // ints, padded to 16 bytes
  // per warp: NB panel buffers, the panels' T^{-1}, the pivot rows
  static constexpr size_t WARP_BYTES = sizeof(double) * ((size_t)NB * PANEL + (size_t)NPAN * 16) + sizeof(int) * PIVS;
  static constexpr size_t DYN = WARP_BYTES * W;
};

// x_e = A_e^{-1} b_e from the Gauss-Jordan record: one warp per cell, lane l
// holds rows l + 32 s of the working vector. Per panel p (in order) the
// pivot rows' values reach every lane by shuffles, t = T_p^{-1} x[pivots],
// and every row takes x_i -= a_i . t with a_i its four panel entries (on a
// pivot row T_r - e_r, which leaves t there): the replay of the elimination
// on one right-hand side. The record reaches shared memory by bulk copies
// (a panel's four columns are one contiguous run of the column-major
// record), NB panels ahead of the replay, each buffer completed on its own
// mbarrier; the panels' T^{-1} and pivot rows arrive with the first panel.
// The record streams once, as an explicit inverse would. The result is in
// pivot order (row w is unknown perm[w]) and is scattered on the way out.
// Waits are bounded: a copy that does not land within kRecSpinLimit polls
// raises DERR_WAIT_LIMIT and the warp returns after a bounded drain of the
// copies it issued (EG_ERR_CONTEXT_LOST when even that runs out).
constexpr unsigned kRecSpinLimit = 1u << 20;
constexpr unsigned kRecDrainLimit = 1u << 24;  // abort path: let an issued copy land
template <int M>
__global__ void __launch_bounds__(32 * RecApplyCfg<M>::W) dg_gj_apply_kernel(
    const double *__restrict__ rec, const double *__restrict__ rec_fac, const int *__restrict__ rec_pivs,
    const int *__restrict__ perm, int nblocks, const double *__restrict__ b, double *__restrict__ x,
    const int *__restrict__ skip, int *err) {
  using C = RecApplyCfg<M>;
  constexpr int S = (M + 31) / 32, NPAN = C::NPAN, NB = C::NB, PANEL = C::PANEL;
  extern __shared__ __align__(16) double dsm[];
  __shared__ __align__(8) unsigned long long bars[C::W][NB];
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * C::W + warp;
  if (blk >= nblocks) return;  // warp-uniform; nothing below synchronises the CTA
  double *buf = reinterpret_cast<double *>(reinterpret_cast<char *>(dsm) + C::WARP_BYTES * warp);
  double *Fs = buf + (size_t)NB * PANEL;
  int *Ps = reinterpret_cast<int *>(Fs + NPAN * 16);
  const double *R = rec + (size_t)blk * M * M;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NB; ++k) mbar_init(&bars[warp][k]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect(&bars[warp][0], (unsigned)(sizeof(double) * (PANEL + NPAN * 16) + sizeof(int) * M));
    bulk_load(Fs, rec_fac + (size_t)blk * NPAN * 16, (unsigned)(sizeof(double) * NPAN * 16), &bars[warp][0]);
    bulk_load(Ps, rec_pivs + (size_t)blk * M, (unsigned)(sizeof(int) * M), &bars[warp][0]);
    bulk_load(buf, R, (unsigned)(sizeof(double) * PANEL), &bars[warp][0]);
#pragma unroll
    for (int k = 1; k < NB; ++k)
      if (k < NPAN) {
        mbar_expect(&bars[warp][k], (unsigned)(sizeof(double) * PANEL));
        bulk_load(buf + (size_t)k * PANEL, R + (size_t)k * PANEL, (unsigned)(sizeof(double) * PANEL), &bars[warp][k]);
      }
  }
  __syncwarp();
  double v[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int i = lane + 32 * s;
    v[s] = i < M ? b[(size_t)blk * M + i] : 0.;
  }
#pragma unroll 1
  for (int p = 0; p < NPAN; ++p) {
    const int k = p % NB;
    const unsigned parity = (unsigned)((p / NB) & 1);
    if (!mbar_wait(&bars[warp][k], parity, kRecSpinLimit)) {
      if (lane == 0) raise_err(err, DERR_WAIT_LIMIT);
      // let the copies already issued land before the warp leaves; if even
      // the longer drain bound runs out, a copy may still write this CTA's
      // shared memory: err[2] tells the host the context can no longer be
      // trusted
      for (int q = p; q < NPAN && q < p + NB; ++q)
        if (!mbar_wait(&bars[warp][q % NB], (unsigned)((q / NB) & 1), kRecDrainLimit) && lane == 0)
          atomicExch(err + 2, 1);
      return;
    }
    const double *pan = buf + (size_t)k * PANEL;
    double xp[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int pr = Ps[4 * p + r];
      double sel = 0.;
#pragma unroll
      for (int s = 0; s < S; ++s)
        if ((pr >> 5) == s) sel = v[s];
      xp[r] = __shfl_sync(0xffffffffu, sel, pr & 31);
    }
    const double *F = Fs + 16 * p;
    double t[4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      t[kk] = F[4 * kk] * xp[0] + F[4 * kk + 1] * xp[1] + F[4 * kk + 2] * xp[2] + F[4 * kk + 3] * xp[3];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int i = lane + 32 * s;
      if (i < M) v[s] -= pan[i] * t[0] + pan[M + i] * t[1] + pan[2 * M + i] * t[2] + pan[3 * M + i] * t[3];
    }
    __syncwarp();  // every lane has read buffer k before it is refilled
    if (lane == 0 && p + NB < NPAN) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect(&bars[warp][k], (unsigned)(sizeof(double) * PANEL));
      bulk_load(buf + (size_t)k * PANEL, R + (size_t)(p + NB) * PANEL, (unsigned)(sizeof(double) * PANEL),
                &bars[warp][k]);
    }
  }
  const int *pb = perm + (size_t)blk * M;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int i = lane + 32 * s;
    if (i < M) x[(size_t)blk * M + pb[i]] = v[s];
  }
}

int sm_count_dginv() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int Q, int WR, int WC, int MINB>
void launch_inverse(Ctx &c, const double *u) {
  using C = GjInvCfg<Q, WR, WC>;
  constexpr size_t dyn = sizeof(double) * (size_t)C::M * C::LD;
  auto kern = dg_inverse_gj_kernel<Q, WR, WC, MINB>;
  if (dyn > 48 * 1024) EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  const int grid = std::min(c.n, sm_count_dginv() * MINB);
  kern<<<grid, C::THREADS, dyn, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u, c.pc_dg,
                                            c.derr);
  EG_CUDA(cudaGetLastError());
}

template <int Q, int MINB, int WR = 2, int WC = 4>
void launch_record(Ctx &c, const double *u) {
  constexpr int M = 4 * Q * Q;
  using C = Gj2Cfg<M, M, WR, WC>;
  if (!c.dg_rec_fac) {
    c.dg_rec_fac = c.alloc_n<double>((size_t)c.n * (M / 4) * 16);
    c.dg_rec_pivs = c.alloc_n<int>((size_t)c.n * M);
  }
  auto kern = dg_gj_record_kernel<Q, MINB, WR, WC>;
  EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::DYN));
  const int grid = std::min(c.n, sm_count_dginv() * MINB);
  kern<<<grid, C::THREADS, C::DYN, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u, c.pc_dg,
                                                c.dg_rec_fac, c.dg_rec_pivs, c.piv_dg, c.derr);
  EG_CUDA(cudaGetLastError());
}

template <int M>
void launch_record_apply(Ctx &c, const double *b, double *x, const int *skip) {
  using C = RecApplyCfg<M>;
  auto kern = dg_gj_apply_kernel<M>;
  EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::DYN));
  kern<<<(c.n + C::W - 1) / C::W, 32 * C::W, C::DYN, c.stream>>>(c.pc_dg, c.dg_rec_fac, c.dg_rec_pivs, c.piv_dg,
                                                                   c.n, b, x, skip, c.derr);
}

void record_apply(Ctx &c, const double *b, double *x, const int *skip) {
  switch (c.q) {
    case 4: launch_record_apply<64>(c, b, x, skip); break;
    case 5: launch_record_apply<100>(c, b, x, skip); break;
    case 6: launch_record_apply<144>(c, b, x, skip); break;
    default: fail(EG_ERR_INVALID, "Gauss-Jordan records cover k = 3..5");
  }
  EG_CUDA(cudaGetLastError());
}

// b = e_col in every cell; inv[e][col][:] = x_e (column col of the cell's inverse)
__global__ void unit_column_kernel(long long n, int M, int col, double *b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n * M; i += (long long)gridDim.x * blockDim.x)
    b[i] = (int)(i % M) == col ? 1. : 0.;
}
__global__ void store_column_kernel(long long n, int M, int col, const double *x, double *inv) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n * M; i += (long long)gridDim.x * blockDim.x)
    inv[(i / M) * M * M + (size_t)col * M + i % M] = x[i];
}

}  // namespace

bool dg_inverse_supported(int q) { return q >= 1 && q <= 6; }
bool dg_pc_is_record(const Ctx &c) { return c.dg_pc_inverse && c.q >= 4 && c.q <= 6; }

void launch_dg_inverse(Ctx &c, const double *u) {
  c.ensure_pc_dg();
  ProfScope ps(c, EG_K_DG_JACOBI, 1);
  switch (c.q) {
    case 1: launch_inverse<1, 1, 1, 8>(c, u); break;
    case 2: launch_inverse<2, 1, 2, 4>(c, u); break;
    case 3: launch_inverse<3, 2, 2, 2>(c, u); break;
    case 4: launch_record<4, 3>(c, u); break;
    case 5: launch_record<5, 2>(c, u); break;
    case 6: launch_record<6, 1, 4, 4>(c, u); break;
    default: fail(EG_ERR_INVALID, "DG block inverses and records support k <= 5");
  }
}

void launch_dg_inverse_apply(Ctx &c, const double *b, double *x) {
  ProfScope ps(c, EG_K_PC_APPLY, 1);
  if (c.q >= 4) {
    record_apply(c, b, x, c.skip);
    return;
  }
  const int grid = (c.n + 7) / 8;
  switch (c.q) {
    case 1: block_inverse_cm_apply_kernel<4><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, nullptr); break;
    case 2: block_inverse_cm_apply_kernel<16><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, nullptr); break;
    case 3: block_inverse_cm_apply_kernel<36><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, nullptr); break;
    default: fail(EG_ERR_INVALID, "explicit DG block inverses cover k <= 2");
  }
  EG_CUDA(cudaGetLastError());
}

void download_dg_record_inverse(Ctx &c, double *dst) {
  const long long n = c.n;
  const int M = c.m;
  double *b = nullptr, *x = nullptr, *inv = nullptr;
  const size_t vec = sizeof(double) * (size_t)n * M;
  if (cudaMalloc(&b, vec) != cudaSuccess || cudaMalloc(&x, vec) != cudaSuccess ||
      cudaMalloc(&inv, vec * M) != cudaSuccess) {
    cudaFree(b);
    cudaFree(x);
    cudaGetLastError();
    fail(EG_ERR_OUT_OF_MEMORY, "no device memory to expand the DG block-Jacobi record");
  }
  const int grid = (int)std::min<long long>((n * M + 255) / 256, 148LL * 16);
  for (int col = 0; col < M; ++col) {
    unit_column_kernel<<<grid, 256, 0, c.stream>>>(n, M, col, b);
    record_apply(c, b, x, nullptr);
    store_column_kernel<<<grid, 256, 0, c.stream>>>(n, M, col, x, inv);
  }
  EG_CUDA(cudaGetLastError());
  const cudaError_t e = cudaMemcpyAsync(dst, inv, vec * M, cudaMemcpyDeviceToHost, c.stream);
  const cudaError_t s = cudaStreamSynchronize(c.stream);
  cudaFree(b);
  cudaFree(x);
  cudaFree(inv);
  if (e != cudaSuccess || s != cudaSuccess) fail(EG_ERR_CUDA, cudaGetErrorString(e != cudaSuccess ? e : s));
}

}  // namespace eg
