// DG block Jacobi as explicit inverses (PartialDGOperator::DiagonalBlocks,
// src/partial.cpp:265-298, factored as in src/linear.cpp:198-202 and applied
// by LinearSolver::Impl::Precondition, src/linear.cpp:66-75).
//
// Factor: each cell's m x m diagonal block is built at the Newton state and
// inverted in place by the blocked Gauss-Jordan of the HDG condensation
// (eg_gj.cuh): 4-column panels, virtual row partial pivoting (the pivots
// LUFactors::Factor would choose), one m8n8k4 FP64 MMA per 8x8 tile and
// panel. In place means the panel's columns, once eliminated, take the unit
// columns e_{pivot row} of the identity the inverse is built from, so every
// panel updates every tile (2 m^3 flops per block instead of the LU's
// 2/3 m^3) and nothing beyond the block is held on chip. The inverse is
// written column-major.
//
// Apply: x_e = A_e^{-1} b_e as a column-major block GEMV, one warp per cell,
// lanes over rows: every load of the inverse is a contiguous 16-byte access
// per lane, so the apply streams the n m^2 doubles once at HBM speed where
// the triangular sweeps of an LU apply are latency bound.
#include <algorithm>

#include "eg_cellmat.cuh"
#include "eg_gj.cuh"
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

// The two-phase form of the same inverse (eg_gj.cuh gj2_reduce/gj2_replay):
// phase 1 reduces the block in shared memory (two or three CTAs of 8 warps
// per SM for k = 3, 4; one CTA of 16 warps for k = 5), phase 2 replays the
// recorded panels on the identity, 16 WC columns per pass. The
// result W has its rows in pivot order -- row w holds row perm[w] of the
// inverse -- and is stored column-major as it leaves the registers; the
// apply scatters through perm.
template <int Q, int MINB, int WR_ = 2, int WC_ = 4>
__global__ void __launch_bounds__(32 * WR_ *WC_, MINB)
    dg_inverse_gj2_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                          double *__restrict__ inv, int *__restrict__ perm, int *err) {
  constexpr int M = 4 * Q * Q;
  using C = Gj2Cfg<M, M, WR_, WC_>;
  constexpr int WR = C::WR, WC = C::WC, TRW = C::TRW, NPAN = C::NPAN, KR = C::KR, NP = C::NP, LDA = C::LDA;
  constexpr int TCB = 2, CBW = 8 * TCB * WC, NPASS = (M + CBW - 1) / CBW;
  __shared__ STab<Q> st;
  __shared__ double us[M], UT[16 * Q], FM[4 * Q * 16];
  __shared__ double topA[4][NP];
  __shared__ double topR[2][4][CBW];
  __shared__ double rowbuf[KR * 32][4];
  __shared__ double fac[NPAN][16];
  __shared__ int pivs[NPAN][4];
  __shared__ int invp[KR * 32];
  __shared__ unsigned char used[KR * 32];
  __shared__ int sing;
  extern __shared__ __align__(16) double A[];
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
    build_cell_matrix<Q>(A, LDA, st, us, FM, g);
    for (int i = threadIdx.x; i < KR * 32; i += C::THREADS) {
      used[i] = i >= M ? 1 : 0;
      invp[i] = 0;
    }
    if (threadIdx.x == 0) sing = 0;
    __syncthreads();
    gj2_reduce<C>(A, topA, rowbuf, fac, pivs, used, invp, &sing);
    double *W = inv + (size_t)e * M * M;
#pragma unroll 1
    for (int pass = 0; pass < NPASS; ++pass) {
      const int c0 = pass * CBW;
      double acc[TRW][TCB][2];
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int row = (wr + a * WR) * 8 + gq;
#pragma unroll
        for (int b = 0; b < TCB; ++b) {
          const int col = c0 + (wc + b * WC) * 8 + 2 * tq;
          acc[a][b][0] = (row < M && col == row) ? 1. : 0.;
          acc[a][b][1] = (row < M && col + 1 == row) ? 1. : 0.;
        }
      }
      gj2_replay<C, TCB>(A, fac, pivs, topR, acc);
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int row = (wr + a * WR) * 8 + gq;
        if (row < M) {
#pragma unroll
          for (int b = 0; b < TCB; ++b) {
            const int col = c0 + (wc + b * WC) * 8 + 2 * tq;
            if (col < M) W[(size_t)col * M + row] = acc[a][b][0];
            if (col + 1 < M) W[(size_t)(col + 1) * M + row] = acc[a][b][1];
          }
        }
      }
      __syncthreads();  // topR is reused by the next pass
    }
    if (sing) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_JACOBI);
      continue;
    }
    for (int i = threadIdx.x; i < M; i += C::THREADS) perm[(size_t)e * M + i] = invp[i];
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
void launch_inverse2(Ctx &c, const double *u) {
  using C = Gj2Cfg<4 * Q * Q, 4 * Q * Q, WR, WC>;
  auto kern = dg_inverse_gj2_kernel<Q, MINB, WR, WC>;
  EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::DYN));
  const int grid = std::min(c.n, sm_count_dginv() * MINB);
  kern<<<grid, C::THREADS, C::DYN, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u, c.pc_dg,
                                                c.piv_dg, c.derr);
  EG_CUDA(cudaGetLastError());
}

}  // namespace

bool dg_inverse_supported(int q) { return q >= 1 && q <= 6; }
bool dg_inverse_permuted(int q) { return q >= 4; }

void launch_dg_inverse(Ctx &c, const double *u) {
  c.ensure_pc_dg();
  ProfScope ps(c, EG_K_DG_JACOBI, 1);
  switch (c.q) {
    case 1: launch_inverse<1, 1, 1, 8>(c, u); break;
    case 2: launch_inverse<2, 1, 2, 4>(c, u); break;
    case 3: launch_inverse<3, 2, 2, 2>(c, u); break;
    case 4: launch_inverse2<4, 3>(c, u); break;
    case 5: launch_inverse2<5, 2>(c, u); break;
    case 6: launch_inverse2<6, 1, 4, 4>(c, u); break;
    default: fail(EG_ERR_INVALID, "explicit DG block inverses support k <= 5");
  }
}

void launch_dg_inverse_apply(Ctx &c, const double *b, double *x) {
  ProfScope ps(c, EG_K_PC_APPLY, 1);
  const int grid = (c.n + 7) / 8;
  const int *perm = dg_inverse_permuted(c.q) ? c.piv_dg : nullptr;
  switch (c.q) {
    case 1: block_inverse_cm_apply_kernel<4><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, perm); break;
    case 2: block_inverse_cm_apply_kernel<16><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, perm); break;
    case 3: block_inverse_cm_apply_kernel<36><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, perm); break;
    case 4: block_inverse_cm_apply_kernel<64><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, perm); break;
    case 5: block_inverse_cm_apply_kernel<100><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, perm); break;
    case 6: block_inverse_cm_apply_kernel<144><<<grid, 256, 0, c.stream>>>(c.pc_dg, c.n, b, x, c.skip, perm); break;
    default: fail(EG_ERR_INVALID, "explicit DG block inverses support k <= 5");
  }
  EG_CUDA(cudaGetLastError());
}

}  // namespace eg
