// Static condensation kernels of the hybridised (HDG) Newton update.
//
// Device layout per cell e (m = 4p, t = 4q):
//   XY[e]      m x (4t+1) column-major: columns 0..4t-1 are X_e = A_e^{-1} B_e,
//              column 4t is y_e = A_e^{-1} r_e  (src/condensation.cpp:131-148);
//   Cb[e]      4q flux blocks C (4x4 column-major) of the face restriction;
//   sf[e]      4q lift scalars of B;
//   contrib[e] 4t face contributions of the last per-cell pass, combined per
//              face by a second pass (two contributions per face, no atomics,
//              deterministic).
#include <algorithm>

#include "eg_cellmat.cuh"
#include "eg_gj.cuh"
#include "eg_internal.h"

namespace eg {

// Shared-memory budget for the dense cell system (227 KB per CTA minus the
// static tables and staging arrays).
constexpr size_t kCellSmemBudget = 200 * 1024;
template <int Q>
__host__ __device__ constexpr int condense_mode() {
  // 0: A and [B|r] in shared memory; 1: A in shared memory, [B|r] in XY;
  // 2: A in a global workspace slab, [B|r] in XY.
  constexpr size_t M = 4 * Q * Q, NR = 16 * Q + 1;
  return sizeof(double) * M * (M + NR) <= kCellSmemBudget ? 0
         : (sizeof(double) * M * M <= kCellSmemBudget ? 1 : 2);
}
template <int Q>
__host__ __device__ constexpr size_t condense_dyn_bytes() {
  constexpr int M = 4 * Q * Q, NR = 16 * Q + 1;
  return condense_mode<Q>() == 0 ? sizeof(double) * (size_t)M * (M + NR)
                                 : (condense_mode<Q>() == 1 ? sizeof(double) * (size_t)M * M : 0);
}

// ---------------------------------------------------------- condensation
// Per-cell staging shared by both condensation kernels.
template <int Q>
struct CondenseShared {
  static constexpr int M = 4 * Q * Q;
  STab<Q> st;
  double us[M], UT[16 * Q], FM[4 * Q * 16], SF[4 * Q], CB[4 * Q * 16];
  int piv_s[M];
  double inv_piv[M];
  double bcast[2];
};

// Assemble the cell system: A (m x m) and [B | r_e] (m x (4t+1)), both
// column-major, A with leading dimension ld and [B | r_e] with ldr (ld when
// not given); also store C and the B scalars.
template <int Q>
__device__ void condense_build(CondenseShared<Q> &sh, const Geo &g, const Frozen &fz,
                               const double *__restrict__ u, const double *__restrict__ r, double *Cb,
                               double *sf_out, double *A, double *R, int e, int ld = 4 * Q * Q, int ldr = -1) {
  if (ldr < 0) ldr = ld;
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
  const STab<Q> &st = sh.st;
  for (int i = threadIdx.x; i < M; i += blockDim.x) sh.us[i] = u[(size_t)e * M + i];
  __syncthreads();
  for (int task = threadIdx.x; task < 4 * Q; task += blockDim.x) {
    const int s = task / Q, j = task % Q;
    double o[4] = {0., 0., 0., 0.};
    for (int l = 0; l < Q; ++l) {
      const double f = st.fb(s, j, l);
      const double *v = sh.us + 4 * line_node<Q>(s, j, l);
#pragma unroll
      for (int c = 0; c < 4; ++c) o[c] += f * v[c];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) sh.UT[task * 4 + c] = o[c];
  }
  __syncthreads();
  // HDG face matrices (src/problem.cpp:661-699): derivative = sign J(U_own)
  // + stab I with stab = a (own left) or b (own right); C = -ew derivative;
  // B lift scalar = -dt len/|K| ew (a or b) (problem.cpp:622-630).
  for (int task = threadIdx.x; task < 4 * Q; task += blockDim.x) {
    const int s = task / Q, j = task % Q;
    const bool L = side_is_left(s);
    const int f = cell_face(e, s, g.nx, g.ny);
    const int fi = f * Q + j;
    const double stab = L ? fz.a[fi] : fz.b[fi];
    double jm[16];
    jacobian(sh.UT + 4 * task, s < 2 ? 0 : 1, g.gm1, jm);
    const double nsign = L ? 1. : -1.;
    const double ewj = st.ew(j);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const double v = nsign * jm[k] + ((k % 5) == 0 ? stab : 0.);
      sh.FM[task * 16 + k] = v;
      const double cv = -ewj * v;
      sh.CB[task * 16 + k] = cv;
      Cb[((size_t)e * 4 * Q + task) * 16 + k] = cv;
    }
    const double len = s < 2 ? g.hy : g.hx;
    const double scale = g.dt * len / g.area * ewj;
    const double sv = -scale * stab;
    sh.SF[task] = sv;
    sf_out[(size_t)e * 4 * Q + task] = sv;
  }
  __syncthreads();
  build_cell_matrix<Q>(A, ld, st, sh.us, sh.FM, g);
  if (R == nullptr) return;  // the caller forms [B | r_e] itself (lift_entry)
  for (int col = threadIdx.x; col < NR; col += blockDim.x) {
    double *rc = R + (size_t)col * ldr;
    if (col < 4 * T) {
      for (int i = 0; i < M; ++i) rc[i] = 0.;
      const int s = col / T, jj = (col % T) >> 2, c = col & 3;
      const double sv = sh.SF[s * Q + jj];
      for (int l = 0; l < Q; ++l) {
        const int i = line_node<Q>(s, jj, l);
        rc[4 * i + c] = st.fb(s, jj, l) * st.inv_mass(i) * sv;
      }
    } else {
      for (int i = 0; i < M; ++i) rc[i] = r[(size_t)e * M + i];
    }
  }
}

// Outputs of a solved cell: X|y to XY (unless already there), rhs
// contributions C_e y_e (src/condensation.cpp:141-142) and the Schur Jacobi
// panels C_s X_s (src/operators.cpp:7-26, 295-301).
template <int Q>
__device__ void condense_epilogue(const CondenseShared<Q> &sh, const double *R, bool copy_out, double *XY,
                                  double *contrib, double *panels, int npan, int e) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
  const STab<Q> &st = sh.st;
  if (copy_out) {
    double *dst = XY + (size_t)e * M * NR;
    for (int i = threadIdx.x; i < M * NR; i += blockDim.x) dst[i] = R[i];
  }
  const double *y = R + (size_t)(4 * T) * M;
  for (int o = threadIdx.x; o < 4 * T; o += blockDim.x) {
    const int s = o / T, jj = (o % T) >> 2, c = o & 3;
    double val[4] = {0., 0., 0., 0.};
    for (int l = 0; l < Q; ++l) {
      const double f = st.fb(s, jj, l);
      const double *yv = y + 4 * line_node<Q>(s, jj, l);
#pragma unroll
      for (int d = 0; d < 4; ++d) val[d] += f * yv[d];
    }
    const double *cb = sh.CB + (s * Q + jj) * 16;
    double res = 0.;
#pragma unroll
    for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * val[d];
    contrib[(size_t)e * 4 * T + o] = res;
  }
  if (panels) {
    // the 4 diagonal panels, or all 16 ([s][o]) where the Schur action uses them
    const bool all16 = npan == 16;
    for (int o = threadIdx.x; o < npan * T * T; o += blockDim.x) {
      const int pan = o / (T * T), rem = o % (T * T);
      const int s = all16 ? pan >> 2 : pan, so = all16 ? pan & 3 : pan;
      const int row = rem % T, cc = rem / T;
      const int jj = row >> 2, c = row & 3;
      const double *xc = R + (size_t)(so * T + cc) * M;
      double val[4] = {0., 0., 0., 0.};
      for (int l = 0; l < Q; ++l) {
        const double f = st.fb(s, jj, l);
        const double *xv = xc + 4 * line_node<Q>(s, jj, l);
#pragma unroll
        for (int d = 0; d < 4; ++d) val[d] += f * xv[d];
      }
      const double *cb = sh.CB + (s * Q + jj) * 16;
      double res = 0.;
#pragma unroll
      for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * val[d];
      panels[(size_t)e * npan * T * T + o] = res;
    }
  }
}

// Entry (row, col) of the lift B (col < 4t) of the cell system: the face
// point's scalar lift sf times phi * inv_mass on the component of the column
// (HybridCell's B, src/problem.cpp:622-630; the same values condense_build
// writes). SF is the cell's staged lift scalars.
template <int Q>
__device__ __forceinline__ double lift_entry(const STab<Q> &st, const double *SF, int row, int col) {
  constexpr int T = 4 * Q;
  const int s = col / T, rem = col % T, jj = rem >> 2, c = rem & 3;
  const int i = row >> 2;
  if ((row & 3) != c) return 0.;
  const int ix = i % Q, iy = i / Q;
  const bool on = s < 2 ? iy == jj : ix == jj;
  if (!on) return 0.;
  const int l = s < 2 ? ix : iy;
  return st.fb(s, jj, l) * st.inv_mass(i) * SF[s * Q + jj];
}

// Outputs of a solved cell from R = [X | y] (stride ldr, unknown order):
// [X | y] to XY (compact), the trace contributions C_e y_e and the Schur
// panels C_s X_o (src/condensation.cpp:141-142, src/operators.cpp:7-26). One
// thread per (side, column) forms the column's trace on the side once
// (q face points x 4 components) and applies the side's 4x4 flux blocks,
// emitting 4q consecutive outputs.
template <int Q>
__device__ void condense_epilogue_traces(const CondenseShared<Q> &sh, const double *R, int ldr, double *XY,
                                         double *contrib, double *panels, int npan, int e) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
  const STab<Q> &st = sh.st;
  double *dst = XY + (size_t)e * M * NR;
  for (int i = threadIdx.x; i < M * NR; i += blockDim.x) dst[i] = R[(size_t)(i / M) * ldr + i % M];
  const bool all16 = npan == 16;
  for (int task = threadIdx.x; task < 4 * NR; task += blockDim.x) {
    const int s = task & 3, col = task >> 2;
    const int so = col / T;  // block column of X (4 = y)
    if (col < 4 * T && !all16 && so != s) continue;
    double *out;
    if (col == 4 * T) {
      out = contrib + (size_t)e * 4 * T + s * T;
    } else {
      if (panels == nullptr) continue;
      const int pan = all16 ? s * 4 + so : s;
      out = panels + (((size_t)e * npan + pan) * T + (col - so * T)) * T;
    }
    const double *xc = R + (size_t)col * ldr;
    for (int jj = 0; jj < Q; ++jj) {
      double v[4] = {0., 0., 0., 0.};
#pragma unroll
      for (int l = 0; l < Q; ++l) {
        const double f = st.fb(s, jj, l);
        const double *xv = xc + 4 * line_node<Q>(s, jj, l);
#pragma unroll
        for (int d = 0; d < 4; ++d) v[d] += f * xv[d];
      }
      const double *cb = sh.CB + (s * Q + jj) * 16;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double res = 0.;
#pragma unroll
        for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * v[d];
        out[jj * 4 + c] = res;
      }
    }
  }
}

// Generic condensation (any degree): CTA-cooperative LU on shared or global
// memory (StreamCondense, src/condensation.cpp:131-148).
template <int Q>
__global__ void __launch_bounds__(256)
    condense_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                    const double *__restrict__ r, double *XY, double *Cb, double *sf_out,
                    double *contrib, double *panels, double *work, int *err) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
  constexpr int MODE = condense_mode<Q>();
  __shared__ CondenseShared<Q> sh;
  extern __shared__ double dyn[];
  load_tables<Q>(sh.st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    double *A = MODE < 2 ? dyn : work + (size_t)blockIdx.x * M * M;
    double *R = MODE == 0 ? dyn + (size_t)M * M : XY + (size_t)e * M * NR;
    condense_build<Q>(sh, g, fz, u, r, Cb, sf_out, A, R, e);
    __syncthreads();
    const bool ok = cta_lu_solve<(M + 31) / 32>(A, M, R, M, M, NR, sh.piv_s, sh.inv_piv, sh.bcast);
    if (!ok) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_CELL);
      continue;
    }
    condense_epilogue<Q>(sh, R, MODE == 0, XY, contrib, panels, g.npan, e);
  }
}

template <int Q, int WR, int WC>
struct GjCfg {
  static constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1, NC = M + NR;
  static constexpr int MT = (M + 7) / 8, NT = (NC + 7) / 8;
  static constexpr int TRW = (MT + WR - 1) / WR, TCW = (NT + WC - 1) / WC;
  static constexpr int MP = 8 * TRW * WR, NP = 8 * TCW * WC;  // padded to whole warp tile grids
  static constexpr int THREADS = 32 * WR * WC;
  static constexpr int LD = M + 1;           // odd staging stride: conflict-free columns
  static constexpr int KR = (M + 31) / 32;   // rows per lane in the pivot search
};


// Blocked Gauss-Jordan condensation on the tensor cores. The augmented cell
// system W = [A | B | r_e] lives in registers as 8x8 accumulator tiles; warp
// (wr, wc) owns tiles (wr + a*WR, wc + b*WC) of a tile grid padded with zero
// rows and columns to whole warp grids. Panels are 4 columns wide:
//  * the 4 pivot rows of panel p publish their trailing columns W_top;
//  * one m8n8k4 MMA per trailing tile applies W_i -= A_i T^{-1} W_top with
//    the A operand A_i = W_i[panel] for ordinary rows and A_i = T_r - e_r for
//    pivot row r, which turns the same MMA into the row normalisation
//    W_r -> (T^{-1} W_top)_r; B fragments T^{-1} W_top are formed per lane;
//  * the tile column holding panel p+1 (always the first trailing one) is
//    staged right after its MMAs, and warp 0 selects the pivots of panel
//    p+1 while the tensor pipe drains the rest of panel p.
// Pivot selection is partial pivoting over the rows not yet used: largest
// magnitude after eliminating the panel's earlier pivots with multipliers
// a_ij * (1/pivot), first row on ties (MFEM LUFactors::Factor), found with
// warp max/min reductions on the IEEE bit pattern. Pivoting is virtual (rows
// never move): after the last panel, row pivrow[j] holds unknown j, so the
// right-hand-side columns hold X_e = A_e^{-1} B_e and y_e = A_e^{-1} r_e,
// permuted back on the way out (StreamCondense, src/condensation.cpp:136-140,
// carried to reduced row echelon form: no triangular solve follows).
template <int Q, int WR, int WC, int MINB>
__global__ void __launch_bounds__(32 * WR *WC, MINB)
    condense_gj_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                       const double *__restrict__ r, double *XY, double *Cb, double *sf_out,
                       double *contrib, double *panels, int *err) {
  using C = GjCfg<Q, WR, WC>;
  constexpr int M = C::M, NC = C::NC, MP = C::MP, NP = C::NP;
  constexpr int TRW = C::TRW, TCW = C::TCW, LD = C::LD, KR = C::KR, NPAN = M / 4;
  __shared__ CondenseShared<Q> sh;
  __shared__ double pan[2][MP][4], top[2][4][NP];
  __shared__ double fac[2][16];   // T^{-1} of the panel's pivot block, row-major 4x4
  __shared__ int pivs[2][4];
  __shared__ int invp[MP];
  __shared__ unsigned char used[MP];
  __shared__ int sing;
  extern __shared__ double dyn[];  // staged system, column-major M x NC, stride LD
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = warp % WR, wc = warp / WR;
  const int gq = lane >> 2, tq = lane & 3;
  load_tables<Q>(sh.st, tab);

  // Warp 0: choose the 4 pivots of the panel staged in pan[buf]; publish
  // T^{-1} and turn the pivot rows of the A operand into T_r - e_r.
  auto select = [&](int jbase, int buf) {
    return gj_select_pivots<M, KR>(jbase, pan[buf], fac[buf], pivs[buf], used, invp, lane);
  };

  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    condense_build<Q>(sh, g, fz, u, r, Cb, sf_out, dyn, dyn + (size_t)LD * M, e, LD);
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
        acc[a][b][0] = (row < M && col < NC) ? dyn[row + (size_t)col * LD] : 0.;
        acc[a][b][1] = (row < M && col + 1 < NC) ? dyn[row + (size_t)(col + 1) * LD] : 0.;
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
    if (warp == 0 && !select(0, 0) && lane == 0) sing = 1;
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < NPAN && !sing; ++p) {
      const int j = 4 * p, pb = p & 1;
      const int pr0 = pivs[pb][0], pr1 = pivs[pb][1], pr2 = pivs[pb][2], pr3 = pivs[pb][3];
      const int tstart = (j + 4) >> 3;  // first tile column holding columns >= j+4 (= panel p+1's)
      // publish the trailing columns of the pivot rows (zero left of j+4)
#pragma unroll
      for (int a = 0; a < TRW; ++a) {
        const int row = (wr + a * WR) * 8 + gq;
        const int rr = row == pr0 ? 0 : row == pr1 ? 1 : row == pr2 ? 2 : row == pr3 ? 3 : -1;
        if (rr >= 0) {
#pragma unroll
          for (int b = 0; b < TCW; ++b) {
            const int tj = wc + b * WC;
            if (tj >= tstart) {
              const int col = tj * 8 + 2 * tq;
              top[pb][rr][col] = col >= j + 4 ? acc[a][b][0] : 0.;
              top[pb][rr][col + 1] = col + 1 >= j + 4 ? acc[a][b][1] : 0.;
            }
          }
        }
      }
      __syncthreads();
      // A operands (row gq, column tq of each tile row) and B operands
      // (row tq, column gq of each tile column) = T^{-1} top
      double af[TRW];
#pragma unroll
      for (int a = 0; a < TRW; ++a) af[a] = -pan[pb][(wr + a * WR) * 8 + gq][tq];
      const double *F = fac[pb];
      const double f0 = F[4 * tq], f1 = F[4 * tq + 1], f2 = F[4 * tq + 2], f3 = F[4 * tq + 3];
      const bool more = p + 1 < NPAN;
      const int jn = j + 4, half = (jn >> 2) & 1, nb = pb ^ 1;
      const bool stager = more && wc == tstart % WC && (tq >> 1) == half;
#pragma unroll
      for (int b = 0; b < TCW; ++b) {
        const int tj = wc + b * WC;
        if (tj >= tstart) {
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
      if (more && warp == 0 && !select(jn, nb) && lane == 0) sing = 1;
      __syncthreads();
    }
    if (sing) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_CELL);
      continue;
    }
    // right-hand sides back to unknown order: R(invp[w], col) = W(w, M + col)
    double *R = dyn;  // compact M x NR, stride M (the staged system is no longer needed)
#pragma unroll
    for (int a = 0; a < TRW; ++a) {
      const int row = (wr + a * WR) * 8 + gq;
      if (row < M) {
        const int jrow = invp[row];
#pragma unroll
        for (int b = 0; b < TCW; ++b) {
          const int col = (wc + b * WC) * 8 + 2 * tq;
          if (col >= M && col < NC) R[(size_t)(col - M) * M + jrow] = acc[a][b][0];
          if (col + 1 >= M && col + 1 < NC) R[(size_t)(col + 1 - M) * M + jrow] = acc[a][b][1];
        }
      }
    }
    __syncthreads();
    condense_epilogue<Q>(sh, R, true, XY, contrib, panels, g.npan, e);
  }
}

// ------------------------------------- two-phase condensation (k = 3..5)
// The cell system [A | B | r_e] of the register-resident kernel above fills
// an SM's register file, so one cell's serial pivot chain leaves the SM idle
// most of the time. This kernel splits the elimination so that two or three
// cells share an SM at k = 3, 4 (CTAs of 8 warps, at most 128 registers per
// thread, one copy of A per CTA in shared memory); at k = 5 A takes 164 KB
// and one CTA of 16 warps fills the SM:
//  1. Gauss-Jordan on A alone, in shared memory, in 4-column panels: warp 0
//     picks the panel's pivots (gj_pick_pivots) and forms T^{-1}
//     (gj_pivot_block_inverse) while the other warps copy the pivot rows'
//     trailing columns; then every warp updates its trailing 8x8 tiles of A
//     with one m8n8k4 FP64 MMA each (W_i -= a_i T^{-1} W_top, a_i = T_r - e_r
//     on pivot rows), loads first, then MMAs, then stores. The panel columns
//     are never touched again: together with T^{-1} and the pivot rows they
//     are the record of the elimination.
//  2. The record is replayed on [B | r_e] held in registers as 8x8 tiles
//     (staged through the cell's own slot of XY, which the epilogue then
//     overwrites with [X | y]): per panel the pivot rows are published and
//     one MMA per tile applies the same update. No search runs in this phase.
// The arithmetic is the register kernel's (the same pivots up to ties
// within 2^-13, 2^-12 at k = 5, the same panel updates), so the results agree with the
// reference's LU solve (src/condensation.cpp:131-148) to rounding.
template <int Q, int MINB, int WR_ = 2, int WC_ = 4>
__global__ void __launch_bounds__(32 * WR_ *WC_, MINB)
    condense_gj2_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                        const double *__restrict__ r, double *XY, double *Cb, double *sf_out, double *contrib,
                        double *panels, int *err) {
  using C = Gj2Cfg<4 * Q * Q, 16 * Q + 1, WR_, WC_>;
  constexpr int M = C::M, NR = C::NR, WR = C::WR, WC = C::WC;
  constexpr int TRW = C::TRW, TCW = C::TCW, NPAN = C::NPAN, KR = C::KR;
  constexpr int NP = C::NP, NQ = C::NQ, LDA = C::LDA;
  __shared__ CondenseShared<Q> sh;
  __shared__ double topA[4][NP];      // pivot rows of A (trailing columns) for the phase-1 update
  __shared__ double topR[2][4][NQ];   // pivot rows of [B | r_e] in phase 2 (double-buffered)
  __shared__ double rowbuf[KR * 32][4];
  __shared__ double fac[NPAN][16];    // T^{-1} of every panel (row-major 4x4)
  __shared__ int pivs[NPAN][4];
  __shared__ int invp[KR * 32];
  __shared__ unsigned char used[KR * 32];
  __shared__ int sing;
  extern __shared__ __align__(16) double A[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = warp % WR, wc = warp / WR;
  const int gq = lane >> 2, tq = lane & 3;
  load_tables<Q>(sh.st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    condense_build<Q>(sh, g, fz, u, r, Cb, sf_out, A, nullptr, e, LDA);
    // [B | r_e] is staged in the cell's slot of XY (L2-resident until
    // [X | y] overwrites it), one element per thread in address order, by
    // the warps that wait while warp 0 searches each panel's pivots: panel p
    // stages the p-th of NPAN slices
    double *Rg = XY + (size_t)e * M * NR;
    const double *re = r + (size_t)e * M;
    const auto stage = [&](int p, int t, int nt) {
      constexpr int SL = (M * NR + NPAN - 1) / NPAN;
      const int end = min(M * NR, (p + 1) * SL);
      for (int i = p * SL + t; i < end; i += nt) {
        const int col = i / M, row = i % M;
        Rg[i] = col == NR - 1 ? re[row] : lift_entry<Q>(sh.st, sh.SF, row, col);
      }
    };
    for (int i = threadIdx.x; i < KR * 32; i += C::THREADS) {
      used[i] = i >= M ? 1 : 0;
      invp[i] = 0;
    }
    if (threadIdx.x == 0) sing = 0;
    __syncthreads();
    // ------------------------------------------------ phase 1: reduce A
    gj2_reduce<C>(A, topA, rowbuf, fac, pivs, used, invp, &sing, stage);
    // ----------------------------- phase 2: replay on [B | r_e] (registers)
    double acc[TRW][TCW][2];
#pragma unroll
    for (int a = 0; a < TRW; ++a) {
      const int row = (wr + a * WR) * 8 + gq;
#pragma unroll
      for (int b = 0; b < TCW; ++b) {
        const int col = (wc + b * WC) * 8 + 2 * tq;
        acc[a][b][0] = (row < M && col < NR) ? Rg[row + (size_t)col * M] : 0.;
        acc[a][b][1] = (row < M && col + 1 < NR) ? Rg[row + (size_t)(col + 1) * M] : 0.;
      }
    }
    gj2_replay<C, TCW>(A, fac, pivs, topR, acc);
    __syncthreads();  // the record in A is no longer read
    if (sing) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_CELL);
      continue;
    }
    // right-hand sides back to unknown order: R(invp[w], col) = W(w, col)
    double *R = A;  // M x NR, odd stride M + 1 (conflict-free column reads in the epilogue)
#pragma unroll
    for (int a = 0; a < TRW; ++a) {
      const int row = (wr + a * WR) * 8 + gq;
      if (row < M) {
        const int jrow = invp[row];
#pragma unroll
        for (int b = 0; b < TCW; ++b) {
          const int col = (wc + b * WC) * 8 + 2 * tq;
          if (col < NR) R[(size_t)col * (M + 1) + jrow] = acc[a][b][0];
          if (col + 1 < NR) R[(size_t)(col + 1) * (M + 1) + jrow] = acc[a][b][1];
        }
      }
    }
    __syncthreads();
    condense_epilogue_traces<Q>(sh, R, M + 1, XY, contrib, panels, g.npan, e);
  }
}

// ------------------------------------------- condensation for k >= 6 (DMMA)
// The cell system [A | B | r_e] (m x (m + 4t + 1)) does not fit on chip for
// k >= 6, so it lives in a per-CTA slab of global memory (L2-resident) and is
// reduced by blocked Gauss-Jordan with virtual partial pivoting in panels of
// GjgCfg::NB columns:
//  1. the panel's columns are staged in shared memory and its pivots chosen
//     column by column exactly as row partial pivoting on the eliminated
//     column would (largest magnitude among rows not yet used, first index on
//     ties: the pivots of LUFactors::Factor, src/condensation.cpp:136-140);
//  2. T = the panel's pivot rows and top = T^-1 W[pivot rows, trailing];
//  3. one rank-NB update W[r, trailing] -= a_r top on the FP64 tensor cores
//     (mma.sync m8n8k4), with a_r the row's panel entries, and T_r - e_r for
//     the panel's own pivot rows, which turns them into the rows of top.
// After the last panel the right-hand-side columns hold X = A^-1 B and
// y = A^-1 r_e in pivot order and are written to XY in unknown order.
template <int Q>
struct GjgCfg {
  static constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1, NC = M + NR;
  static constexpr int NB = 16;                      // panel width
  static constexpr int NPAN = (M + NB - 1) / NB;
  static constexpr int MT = (M + 7) / 8;            // 8-row tiles
  static constexpr int RU = 6;                       // row tiles per load round of the update
  static constexpr size_t SMEM = sizeof(double) * ((size_t)2 * NB * M + (size_t)NB * NC + 2 * NB * NB) +
                                 sizeof(int) * (size_t)(3 * M + NB);
  // two CTAs per SM where their shared memory fits (k = 6): one CTA's
  // serial pivot chain then overlaps the other's trailing update
  static constexpr int MINB =
      2 * (SMEM + sizeof(CondenseShared<Q>) + 2048) <= 227 * 1024 ? 2 : 1;
};

template <int Q>
__global__ void __launch_bounds__(256, GjgCfg<Q>::MINB)
    condense_gjg_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                        const double *__restrict__ r, double *XY, double *Cb, double *sf, double *contrib,
                        double *panels, double *work, int *err) {
  using C = GjgCfg<Q>;
  constexpr int M = C::M, NR = C::NR, NC = C::NC, NB = C::NB;
  __shared__ CondenseShared<Q> sh;
  __shared__ int sing;
  __shared__ double pivval;
  extern __shared__ __align__(16) double dyn[];
  double *P0 = dyn;                          // original panel columns  [NB][M]
  double *Pw = P0 + (size_t)NB * M;          // working panel columns   [NB][M]
  double *top = Pw + (size_t)NB * M;         // [NB][NC] (trailing width)
  double *Tm = top + (size_t)NB * NC;        // [NB][2NB] augmented [T | I], row-major
  int *used = reinterpret_cast<int *>(Tm + 2 * NB * NB);
  int *pidx = used + M;                      // panel index of a pivot row of this panel, else -1
  int *piv = pidx + M;                       // pivot row of every column
  int *prow = piv + M;                       // pivot rows of this panel
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  double *W = work + (size_t)blockIdx.x * M * NC;  // column-major, ld M
  load_tables<Q>(sh.st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    condense_build<Q>(sh, g, fz, u, r, Cb, sf, W, W + (size_t)M * M, e, M);
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      used[i] = 0;
      pidx[i] = -1;
    }
    if (threadIdx.x == 0) sing = 0;
    __syncthreads();
    for (int pan = 0; pan < C::NPAN; ++pan) {
      const int c0 = pan * NB, nb = min(NB, M - c0), cs = c0 + nb, ntr = NC - cs;
      // 1. stage the panel; choose its pivots on a working copy
      for (int o = threadIdx.x; o < NB * M; o += blockDim.x) {
        const int j = o / M, rr = o % M;
        const double v = j < nb ? W[(size_t)(c0 + j) * M + rr] : 0.;
        P0[o] = v;
        Pw[o] = v;
      }
      __syncthreads();
      for (int j = 0; j < nb; ++j) {
        if (warp == 0) {
          // largest |Pw[j][r]| among unused rows, first row on ties, NaN never
          // chosen: magnitudes compared as IEEE bit patterns (integer compares,
          // three warp reductions)
          constexpr unsigned long long kAbs = 0x7fffffffffffffffull, kInf = 0x7ff0000000000000ull;
          unsigned long long best = 0ull;
          int bi = M;
          for (int rr = lane; rr < M; rr += 32) {
            if (used[rr]) continue;
            const unsigned long long bits =
                (unsigned long long)__double_as_longlong(Pw[(size_t)j * M + rr]) & kAbs;
            if (bits <= kInf && (bi == M || bits > best)) {
              best = bits;
              bi = rr;
            }
          }
          const unsigned hi = (unsigned)(best >> 32), lo = (unsigned)best;
          const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
          const bool c1 = bi < M && hi == mhi;
          const unsigned mlo = __reduce_max_sync(0xffffffffu, c1 ? lo : 0u);
          bi = (int)__reduce_min_sync(0xffffffffu, c1 && lo == mlo ? (unsigned)bi : (unsigned)M);
          if (lane == 0) {
            const double pv = bi < M ? Pw[(size_t)j * M + bi] : 0.;  // an all-NaN column is singular
            if (!(fabs(pv) > 0.)) {
              sing = 1;
              bi = 0;
            }
            pivval = pivot_reciprocal(pv);
            prow[j] = bi;
            piv[c0 + j] = bi;
            used[bi] = 1;
            pidx[bi] = j;
          }
        }
        __syncthreads();
        if (sing) break;
        const int pr = prow[j];
        const double inv = pivval;  // 1 / pivot
        const int rest = nb - j - 1;
        for (int o = threadIdx.x; o < rest * M; o += blockDim.x) {
          const int jj = j + 1 + o / M, rr = o % M;
          if (rr != pr) Pw[(size_t)jj * M + rr] -= Pw[(size_t)j * M + rr] * inv * Pw[(size_t)jj * M + pr];
        }
        __syncthreads();
      }
      if (sing) break;
      // 2. T^-1 by Gauss-Jordan with partial pivoting on [T | I] (nb x 2nb)
      for (int o = threadIdx.x; o < NB * 2 * NB; o += blockDim.x) {
        const int i = o / (2 * NB), k = o % (2 * NB);
        double v = 0.;
        if (i < nb && k < nb) v = P0[(size_t)k * M + prow[i]];
        else if (k >= NB && k - NB == i) v = 1.;
        else if (i >= nb && k == i) v = 1.;  // identity padding of a partial panel
        Tm[o] = v;
      }
      __syncthreads();
      if (warp == 0) {
        for (int j = 0; j < NB; ++j) {
          // pivot among rows j..NB-1 of column j (lane i holds row i): largest
          // magnitude, first row on ties, NaN never chosen (row j if all are)
          constexpr unsigned long long kAbs = 0x7fffffffffffffffull, kInf = 0x7ff0000000000000ull;
          const unsigned long long bits =
              lane < NB ? (unsigned long long)__double_as_longlong(Tm[lane * 2 * NB + j]) & kAbs : 0ull;
          const bool cand = lane >= j && lane < NB && bits <= kInf;
          const unsigned hi = cand ? (unsigned)(bits >> 32) : 0u, lo = cand ? (unsigned)bits : 0u;
          const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
          const bool c1 = cand && hi == mhi;
          const unsigned mlo = __reduce_max_sync(0xffffffffu, c1 ? lo : 0u);
          const unsigned first = __reduce_min_sync(0xffffffffu, c1 && lo == mlo ? (unsigned)lane : 32u);
          const int bi = first < 32u ? (int)first : j;
          const double pv = Tm[bi * 2 * NB + j];
          __syncwarp();
          if (bi != j) {  // swap rows j and bi (lane = column)
            const double a0 = Tm[j * 2 * NB + lane], b0 = Tm[bi * 2 * NB + lane];
            __syncwarp();
            Tm[j * 2 * NB + lane] = b0;
            Tm[bi * 2 * NB + lane] = a0;
          }
          __syncwarp();
          const double ip = 1.0 / pv;
          Tm[j * 2 * NB + lane] *= ip;
          __syncwarp();
          double f[NB];
#pragma unroll
          for (int i = 0; i < NB; ++i) f[i] = Tm[i * 2 * NB + j];
          __syncwarp();
#pragma unroll
          for (int i = 0; i < NB; ++i)
            if (i != j) Tm[i * 2 * NB + lane] -= f[i] * Tm[j * 2 * NB + lane];
          __syncwarp();
        }
      }
      // top = T^-1 W[prow, trailing]: gather the pivot rows, then transform in place
      for (int o = threadIdx.x; o < NB * ntr; o += blockDim.x) {
        const int k = o / ntr, c = o % ntr;
        top[(size_t)k * NC + c] = k < nb ? W[(size_t)(cs + c) * M + prow[k]] : 0.;
      }
      __syncthreads();
      for (int c = threadIdx.x; c < ntr; c += blockDim.x) {
        double wv[NB], out[NB];
#pragma unroll
        for (int k = 0; k < NB; ++k) wv[k] = top[(size_t)k * NC + c];
#pragma unroll
        for (int i = 0; i < NB; ++i) {
          double s = 0.;
#pragma unroll
          for (int k = 0; k < NB; ++k) s += Tm[i * 2 * NB + NB + k] * wv[k];
          out[i] = s;
        }
#pragma unroll
        for (int i = 0; i < NB; ++i) top[(size_t)i * NC + c] = i < nb ? out[i] : 0.;
      }
      __syncthreads();
      // 3. rank-NB update of the trailing columns on the tensor cores
      const int ntile_c = (ntr + 7) / 8;
      for (int ct = warp; ct < ntile_c; ct += nwarps) {
        double bf[NB / 4];
#pragma unroll
        for (int ks = 0; ks < NB / 4; ++ks) {
          const int cc = ct * 8 + gq;
          bf[ks] = cc < ntr ? top[(size_t)(4 * ks + tq) * NC + cc] : 0.;
        }
        const int col0 = cs + ct * 8 + 2 * tq;
        const bool ok0 = col0 < NC, ok1 = col0 + 1 < NC;
        // GjgCfg::RU row tiles per round: their loads are all in flight before the MMAs
        for (int rt0 = 0; rt0 < C::MT; rt0 += C::RU) {
          double cv[C::RU][2];
#pragma unroll
          for (int u = 0; u < C::RU; ++u) {
            const int ra = (rt0 + u) * 8 + gq;  // row of this lane's A fragment and C values
            const bool rok = ra < M;
            cv[u][0] = rok && ok0 ? W[(size_t)col0 * M + ra] : 0.;
            cv[u][1] = rok && ok1 ? W[(size_t)(col0 + 1) * M + ra] : 0.;
          }
#pragma unroll
          for (int u = 0; u < C::RU; ++u) {
            const int ra = (rt0 + u) * 8 + gq;
            const bool rok = ra < M;
            const int pi = rok ? pidx[ra] : -1;
#pragma unroll
            for (int ks = 0; ks < NB / 4; ++ks) {
              const int k = 4 * ks + tq;
              double a = rok ? P0[(size_t)k * M + ra] : 0.;
              if (pi == k) a -= 1.;
              dmma_m8n8k4(cv[u][0], cv[u][1], -a, bf[ks]);
            }
          }
#pragma unroll
          for (int u = 0; u < C::RU; ++u) {
            const int ra = (rt0 + u) * 8 + gq;
            if (ra < M && ok0) W[(size_t)col0 * M + ra] = cv[u][0];
            if (ra < M && ok1) W[(size_t)(col0 + 1) * M + ra] = cv[u][1];
          }
        }
      }
      __syncthreads();  // every warp has finished reading pidx for this panel
      for (int j = threadIdx.x; j < nb; j += blockDim.x) pidx[prow[j]] = -1;
      __syncthreads();
    }
    if (sing) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_CELL);
      continue;
    }
    // right-hand sides back to unknown order: X(j, c) = W(piv[j], M + c)
    double *R = XY + (size_t)e * M * NR;
    for (int o = threadIdx.x; o < M * NR; o += blockDim.x) {
      const int c = o / M, j = o % M;
      R[o] = W[(size_t)(M + c) * M + piv[j]];
    }
    __syncthreads();
    condense_epilogue<Q>(sh, R, false, XY, contrib, panels, g.npan, e);
  }
}

// -------------------------------------------------- Schur action / recovery
// Per cell: gather the 4t trace values, mid = X_e v_e (GEMV streaming X once),
// then either restrict with C (Schur action, src/operators.cpp:166-178) or
// write du = -mid - y (Recover, src/condensation.cpp:28-41, 154-163).
template <int Q, bool RECOVER>
__global__ void __launch_bounds__(128)
    cell_gemv_kernel(Geo g, const double *__restrict__ tab, const double *__restrict__ XY,
                     const double *__restrict__ Cb, const double *__restrict__ v,
                     double *__restrict__ out, const int *__restrict__ skip) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  __shared__ STab<Q> st;
  __shared__ double vl[4 * T], mid[M];
  load_tables<Q>(st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * T; i += blockDim.x) {
      const int s = i / T;
      vl[i] = v[(size_t)cell_face(e, s, g.nx, g.ny) * T + (i % T)];
    }
    __syncthreads();
    const double *X = XY + (size_t)e * M * NR;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      double acc = 0.;
#pragma unroll 8
      for (int col = 0; col < 4 * T; ++col) acc += X[(size_t)col * M + i] * vl[col];
      if (RECOVER) {
        out[(size_t)e * M + i] = -acc - X[(size_t)(4 * T) * M + i];
      } else {
        mid[i] = acc;
      }
    }
    if (!RECOVER) {
      __syncthreads();
      for (int o = threadIdx.x; o < 4 * T; o += blockDim.x) {
        const int s = o / T, jj = (o % T) >> 2, c = o & 3;
        double val[4] = {0., 0., 0., 0.};
        for (int l = 0; l < Q; ++l) {
          const double f = st.fb(s, jj, l);
          const double *mv = mid + 4 * line_node<Q>(s, jj, l);
#pragma unroll
          for (int d = 0; d < 4; ++d) val[d] += f * mv[d];
        }
        const double *cb = Cb + ((size_t)e * 4 * Q + s * Q + jj) * 16;
        double res = 0.;
#pragma unroll
        for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * val[d];
        out[(size_t)e * 4 * T + o] = res;
      }
    }
  }
}

// Schur action from the 16 panels of a cell (degrees with
// schur_panels_full, and every degree with element or full assembly, where the
// panels are the element entries C X of src/condensation.cpp:143-146):
// contrib[e][s] = sum_o (C_s X_o) v_o, the same product as the C restriction
// of X v (src/operators.cpp:166-178) with the C X panels formed once per
// condensation, so that each apply streams 16 t^2 doubles per cell instead of
// m x 4t. One thread per output (s, row); consecutive rows read consecutive
// panel entries.
template <int Q>
__global__ void __launch_bounds__(((16 * Q + 31) / 32) * 32)
    panel_gemv_kernel(Geo g, const double *__restrict__ panels, const double *__restrict__ v,
                      double *__restrict__ out, const int *__restrict__ skip) {
  constexpr int T = 4 * Q, TT = T * T;
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  __shared__ double vl[4 * T];
  const int o = threadIdx.x, s = o / T, row = o % T;
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * T; i += blockDim.x)
      vl[i] = v[(size_t)cell_face(e, i / T, g.nx, g.ny) * T + (i % T)];
    __syncthreads();
    if (o < 4 * T) {
      const double *P = panels + ((size_t)e * 16 + s * 4) * TT + row;
      double acc = 0.;
#pragma unroll 8
      for (int k = 0; k < 4 * T; ++k) acc += P[(size_t)(k / T) * TT + (k % T) * T] * vl[k];
      out[(size_t)e * 4 * T + o] = acc;
    }
  }
}

// y_f = D_f v_f - contrib[L][ls] - contrib[R][rs]  (one thread per trace dof)
__global__ void face_combine_kernel(int nx, int ny, int T, int nl, const double *__restrict__ D,
                                    const double *__restrict__ v, const double *__restrict__ contrib,
                                    double sign_v, double *__restrict__ y, const int *__restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nl) return;
  const int f = idx / T, i = idx % T;
  const int L = f >> 1, ls = (f & 1) ? 3 : 1;
  const int R = neighbour(L, ls, nx, ny), rs = ls - 1;
  const double base = D ? D[idx] * v[idx] : 0.;
  y[idx] = sign_v * ((base - contrib[(size_t)L * 4 * T + ls * T + i]) -
                     contrib[(size_t)R * 4 * T + rs * T + i]);
}

// er = -B (eq / D) (RecoveredResidual, src/stepper.cpp:10-26); one thread per
// (cell, node).
template <int Q>
__global__ void __launch_bounds__(256)
    recovered_residual_kernel(Geo g, const double *__restrict__ tab, const double *__restrict__ sf,
                              const double *__restrict__ D, const double *__restrict__ eq,
                              double *__restrict__ er) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q;
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.n * P) return;
  const int e = idx / P, node = idx % P, ix = node % Q, iy = node / Q;
  const double im = st.inv_mass(node);
  double acc[4] = {0., 0., 0., 0.};
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int j = s < 2 ? iy : ix, l = s < 2 ? ix : iy;
    const int f = cell_face(e, s, g.nx, g.ny);
    const double wgt = st.fb(s, j, l) * im;
    const double a = sf[(size_t)e * 4 * Q + s * Q + j];
    const size_t base = (size_t)f * T + 4 * j;
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += wgt * (a * (eq[base + c] / D[base + c]));
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) er[(size_t)e * M + 4 * node + c] = -acc[c];
}

// Schur block-Jacobi: S_ff = D_f - P_L - P_R (ElementOperator::DiagonalBlocks
// src/operators.cpp:275-303). With factor set, the block is inverted through
// its pivoted LU (LUFactors, src/linear.cpp:198-202) applied to the identity,
// and the explicit inverse is stored so the preconditioner apply is a
// coalesced batched GEMV instead of two dependent triangular sweeps.
template <int T>
__global__ void __launch_bounds__(64)
    schur_jacobi_kernel(int nx, int ny, int nf, int npan, const double *__restrict__ D,
                        const double *__restrict__ panels, double *blocks, int *pivots, bool factor,
                        int *err) {
  __shared__ double S[T * T], Inv[T * T];
  __shared__ int piv_s[T];
  __shared__ double inv_piv[T];
  __shared__ double bcast[2];
  for (int f = blockIdx.x; f < nf; f += gridDim.x) {
    __syncthreads();
    const int L = f >> 1, ls = (f & 1) ? 3 : 1;
    const int R = neighbour(L, ls, nx, ny), rs = ls - 1;
    // diagonal panels C_s X_s of the two cells (panel s*5 of 16 where all are kept)
    const bool all16 = npan == 16;
    const double *pl = panels + (all16 ? (size_t)L * 16 + ls * 5 : (size_t)L * 4 + ls) * T * T;
    const double *pr = panels + (all16 ? (size_t)R * 16 + rs * 5 : (size_t)R * 4 + rs) * T * T;
    for (int o = threadIdx.x; o < T * T; o += blockDim.x) {
      const int row = o % T, col = o / T;
      const double d = row == col ? D[(size_t)f * T + row] : 0.;
      S[o] = (d - pl[o]) - pr[o];
      Inv[o] = row == col ? 1. : 0.;
    }
    __syncthreads();
    const double *out = S;
    if (factor) {
      const bool ok = cta_lu_solve<(T + 31) / 32>(S, T, Inv, T, T, T, piv_s, inv_piv, bcast);
      if (!ok && threadIdx.x == 0) raise_err(err, DERR_SINGULAR_JACOBI);
      out = Inv;
    }
    for (int i = threadIdx.x; i < T; i += blockDim.x) pivots[(size_t)f * T + i] = factor ? piv_s[i] : i;
    // stored row-major (one contiguous row per output of the block GEMV)
    for (int o = threadIdx.x; o < T * T; o += blockDim.x) blocks[(size_t)f * T * T + (o % T) * T + o / T] = out[o];
  }
}

// The same blocks inverted by one warp per face for T <= 32: lane r holds row
// r of [S | I] in registers and Gauss-Jordan runs with partial pivoting over
// the rows not yet used as pivot rows (largest magnitude, first row on ties,
// NaN never chosen; a zero pivot is singular, as in LU with row exchanges).
// Rows never move: the pivot row of step k ends up holding row k of S^{-1}.
// The pivot search is three warp reductions on IEEE bit patterns and the
// normalised pivot row is broadcast by shuffles, so no step needs a barrier.
// `pivots` receives the pivot row of every step. Blocks are stored row-major.
template <int T>
__global__ void __launch_bounds__(128)
    schur_jacobi_warp_kernel(int nx, int ny, int nf, int npan, const double *__restrict__ D,
                             const double *__restrict__ panels, double *blocks, int *pivots, bool factor,
                             int *err) {
  static_assert(T <= 32, "one row per lane");
  constexpr unsigned long long kAbs = 0x7fffffffffffffffull, kInf = 0x7ff0000000000000ull;
  const int lane = threadIdx.x & 31;
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int f = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); f < nf; f += nwarps) {
    const int L = f >> 1, ls = (f & 1) ? 3 : 1;
    const int R = neighbour(L, ls, nx, ny), rs = ls - 1;
    // diagonal panels C_s X_s of the two cells (panel s*5 of 16 where all are kept)
    const bool all16 = npan == 16;
    const double *pl = panels + (all16 ? (size_t)L * 16 + ls * 5 : (size_t)L * 4 + ls) * T * T;
    const double *pr = panels + (all16 ? (size_t)R * 16 + rs * 5 : (size_t)R * 4 + rs) * T * T;
    const bool row_ok = lane < T;
    const double d = row_ok ? D[(size_t)f * T + lane] : 0.;
    double sr[T], xr[T];
#pragma unroll
    for (int c = 0; c < T; ++c) {
      sr[c] = row_ok ? ((lane == c ? d : 0.) - pl[c * T + lane]) - pr[c * T + lane] : 0.;
      xr[c] = lane == c ? 1. : 0.;
    }
    double *out = blocks + (size_t)f * T * T;  // row-major
    if (!factor) {
      if (row_ok) {
#pragma unroll
        for (int c = 0; c < T; ++c) out[lane * T + c] = sr[c];
        pivots[(size_t)f * T + lane] = lane;
      }
      continue;
    }
    bool un = row_ok;
    int pos = 0;
    bool singular = false;
#pragma unroll
    for (int k = 0; k < T; ++k) {
      double sk = 0.;
#pragma unroll
      for (int c = 0; c < T; ++c)
        if (c == k) sk = sr[c];
      const unsigned long long bits = (unsigned long long)__double_as_longlong(sk) & kAbs;
      const bool cand = un && bits <= kInf;
      const unsigned hi = cand ? (unsigned)(bits >> 32) : 0u, lo = cand ? (unsigned)bits : 0u;
      const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
      const bool c1 = cand && hi == mhi;
      const unsigned mlo = __reduce_max_sync(0xffffffffu, c1 ? lo : 0u);
      const unsigned pw = __reduce_min_sync(0xffffffffu, c1 && lo == mlo ? (unsigned)lane : 32u);
      // a zero pivot (warp-uniform) marks the block singular; the remaining
      // steps run on row 0 and their results are discarded
      const bool zero = pw >= 32u || (mhi == 0u && mlo == 0u);
      singular = singular || zero;
      const int p = zero ? 0 : (int)pw;
      const double l = sk;
      const double ip = 1.0 / __shfl_sync(0xffffffffu, l, p);
      const bool me = lane == p;
#pragma unroll
      for (int c = 0; c < T; ++c) {
        if (c > k) {
          const double v = __shfl_sync(0xffffffffu, sr[c], p) * ip;
          sr[c] = me ? v : sr[c] - l * v;
        }
      }
#pragma unroll
      for (int c = 0; c < T; ++c) {
        const double v = __shfl_sync(0xffffffffu, xr[c], p) * ip;
        xr[c] = me ? v : xr[c] - l * v;
      }
#pragma unroll
      for (int c = 0; c < T; ++c)
        if (c == k) sr[c] = me ? 1. : 0.;
      if (me) {
        un = false;
        pos = k;
      }
    }
    if (singular) {
      if (lane == 0) raise_err(err, DERR_SINGULAR_JACOBI);
      continue;
    }
    if (row_ok) {
#pragma unroll
      for (int c = 0; c < T; ++c) out[pos * T + c] = xr[c];
      pivots[(size_t)f * T + pos] = lane;
    }
  }
}

// x_b = Inv_b b_b for row-major bs x bs inverses (bs even); one thread per
// output row, which reads its row with 16-byte loads. BS > 0 fixes the block
// size at compile time, so the row loop unrolls and all of a row's loads are
// in flight together (BS = 0: any even size).
template <int BS>
__global__ void __launch_bounds__(256) block_gemv_kernel(const double *__restrict__ inv, int nblocks, int bs_rt,
                                                         const double *__restrict__ b,
                                                         double *__restrict__ x, const int *__restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int bs = BS > 0 ? BS : bs_rt;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (long long)nblocks * bs) return;
  const int blk = (int)(id / bs);
  const double2 *ib = reinterpret_cast<const double2 *>(inv + (size_t)id * bs);
  const double *bb = b + (size_t)blk * bs;
  double acc = 0.;
#pragma unroll
  for (int c = 0; c < (BS > 0 ? BS / 2 : bs / 2); ++c) {
    const double2 a = ib[c];
    acc += a.x * bb[2 * c];
    acc += a.y * bb[2 * c + 1];
  }
  x[id] = acc;
}

// In-place transpose of every bs x bs block (one thread per pair i < j).
__global__ void transpose_blocks_kernel(double *a, int nblocks, int bs) {
  const long long per = (long long)bs * (bs - 1) / 2;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= per * nblocks) return;
  const int blk = (int)(id / per);
  int k = (int)(id % per), i = 0;
  while (k >= bs - 1 - i) {  // row i holds the pairs (i, i+1..bs-1)
    k -= bs - 1 - i;
    ++i;
  }
  const int j = i + 1 + k;
  double *m = a + (size_t)blk * bs * bs;
  const double t = m[i * bs + j];
  m[i * bs + j] = m[j * bs + i];
  m[j * bs + i] = t;
}

// ================================================================ launchers
static int sm_count_hdg() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

static int condense_grid(Ctx &c) { return std::min(c.n, sm_count_hdg() * 4); }

template <int Q, int WR, int WC, int MINB>
static void launch_condense_gj(Ctx &c, const double *u, const double *r) {
  using C = GjCfg<Q, WR, WC>;
  constexpr size_t dyn = sizeof(double) * (size_t)C::LD * C::NC;
  auto kern = condense_gj_kernel<Q, WR, WC, MINB>;
  if (dyn > 48 * 1024)
    EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  const int grid = std::min(c.n, sm_count_hdg() * MINB);
  kern<<<grid, C::THREADS, dyn, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u, r,
                                            c.XY, c.Cb, c.sf, c.contrib, c.panels, c.derr);
}

template <int Q, int MINB, int WR = 2, int WC = 4>
static void launch_condense_gj2(Ctx &c, const double *u, const double *r) {
  using C = Gj2Cfg<4 * Q * Q, 16 * Q + 1, WR, WC>;
  auto kern = condense_gj2_kernel<Q, MINB, WR, WC>;
  EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::DYN));
  const int grid = std::min(c.n, sm_count_hdg() * MINB);
  kern<<<grid, C::THREADS, C::DYN, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u, r,
                                                c.XY, c.Cb, c.sf, c.contrib, c.panels, c.derr);
}

template <int Q>
static void launch_condense_gjg(Ctx &c, const double *u, const double *r) {
  using C = GjgCfg<Q>;
  auto kern = condense_gjg_kernel<Q>;
  EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
  int per_sm = 0;
  EG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, C::SMEM));
  const int grid = std::min(c.n, std::max(1, std::min(per_sm, C::MINB)) * sm_count_hdg());
  if (c.work_gj == nullptr || c.work_gj_slots < grid) {
    c.work_gj = c.alloc_n<double>((size_t)grid * C::M * C::NC);
    c.work_gj_slots = grid;
  }
  kern<<<grid, 256, C::SMEM, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u, r, c.XY,
                                          c.Cb, c.sf, c.contrib, c.panels, c.work_gj, c.derr);
}

void launch_condense(Ctx &c, const double *u, const double *r) {
  c.ensure_hdg();
  const int grid = condense_grid(c);
  ProfScope ps(c, EG_K_CONDENSE, 2);
  switch (c.q) {
    case 1: launch_condense_gj<1, 1, 1, 8>(c, u, r); break;
    case 2: launch_condense_gj<2, 1, 2, 6>(c, u, r); break;
    case 3: launch_condense_gj<3, 2, 2, 4>(c, u, r); break;
    case 4: launch_condense_gj2<4, 3>(c, u, r); break;
    case 5: launch_condense_gj2<5, 2>(c, u, r); break;
    case 6: launch_condense_gj2<6, 1, 4, 4>(c, u, r); break;
    case 7: launch_condense_gjg<7>(c, u, r); break;
    case 8: launch_condense_gjg<8>(c, u, r); break;
    case 9: launch_condense_gjg<9>(c, u, r); break;
    default:
      EG_DISPATCH_Q(c.q, {
        constexpr size_t dyn = condense_dyn_bytes<Q>();
        auto kern = condense_kernel<Q>;
        if (dyn > 48 * 1024)
          EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        if (condense_mode<Q>() == 2 && (c.work_cell == nullptr || c.work_slots < grid)) {
          constexpr int M = 4 * Q * Q;
          c.work_cell = c.alloc_n<double>((size_t)grid * M * M);
          c.work_slots = grid;
        }
        kern<<<grid, 256, dyn, c.stream>>>(c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, u,
                                           r, c.XY, c.Cb, c.sf, c.contrib, c.panels, c.work_cell,
                                           c.derr);
      });
  }
  EG_CUDA(cudaGetLastError());
  // rhs_f = contrib_L + contrib_R (s.rhs = 0; rhs[ids] += C y)
  const int blocks = (c.nl + 255) / 256;
  face_combine_kernel<<<blocks, 256, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.t, c.nl, nullptr, c.rhs,
                                                    c.contrib, -1.0, c.rhs, nullptr);
  EG_CUDA(cudaGetLastError());
  c.condensed = true;
}

void launch_schur_apply(Ctx &c, const double *v, double *y) {
  ProfScope ps(c, EG_K_SCHUR_APPLY, 2);
  const int grid = std::min(c.n, sm_count_hdg() * 16);
  if (c.geo.npan == 16) {
    switch (c.q) {
#define EG_PG(QQ)                                                                                          \
  case QQ:                                                                                                 \
    panel_gemv_kernel<QQ><<<grid, ((16 * QQ + 31) / 32) * 32, 0, c.stream>>>(c.geo, c.panels, v, c.contrib, \
                                                                            c.skip);                       \
    break;
      EG_PG(1) EG_PG(2) EG_PG(3) EG_PG(4) EG_PG(5) EG_PG(6) EG_PG(7) EG_PG(8) EG_PG(9)
#undef EG_PG
      default:
        fail(EG_ERR_INVALID, "unsupported degree");
    }
  } else {
    EG_DISPATCH_Q(c.q, (cell_gemv_kernel<Q, false><<<grid, 128, 0, c.stream>>>(c.geo, c.tab, c.XY, c.Cb,
                                                                              v, c.contrib, c.skip)));
  }
  EG_CUDA(cudaGetLastError());
  const int blocks = (c.nl + 255) / 256;
  face_combine_kernel<<<blocks, 256, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.t, c.nl, c.D, v,
                                                    c.contrib, 1.0, y, c.skip);
  EG_CUDA(cudaGetLastError());
}

void launch_recover(Ctx &c, const double *lam, double *du) {
  ProfScope ps(c, EG_K_RECOVER, 1);
  const int grid = std::min(c.n, sm_count_hdg() * 16);
  EG_DISPATCH_Q(c.q, (cell_gemv_kernel<Q, true><<<grid, 128, 0, c.stream>>>(c.geo, c.tab, c.XY, c.Cb,
                                                                           lam, du, nullptr)));
  EG_CUDA(cudaGetLastError());
}

void launch_recovered_residual(Ctx &c, const double *eq, double *er) {
  const int total = c.n * c.p;
  ProfScope ps(c, EG_K_RECOVERED_RESIDUAL, 1);
  EG_DISPATCH_Q(c.q, (recovered_residual_kernel<Q><<<(total + 255) / 256, 256, 0, c.stream>>>(
                         c.geo, c.tab, c.sf, c.D, eq, er)));
  EG_CUDA(cudaGetLastError());
}

void launch_transpose_blocks(Ctx &c, double *a, int nblocks, int bs) {
  const long long total = (long long)nblocks * bs * (bs - 1) / 2;
  if (total == 0) return;
  transpose_blocks_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(a, nblocks, bs);
  EG_CUDA(cudaGetLastError());
}

void launch_block_inverse_apply(Ctx &c, const double *inv, int nblocks, int bs, const double *b, double *x) {
  ProfScope ps(c, EG_K_PC_APPLY, 1);
  const long long total = (long long)nblocks * bs;
  const unsigned grid = (unsigned)((total + 255) / 256);
  switch (bs) {
#define EG_BG(BB)                                                                                  \
  case BB:                                                                                         \
    block_gemv_kernel<BB><<<grid, 256, 0, c.stream>>>(inv, nblocks, bs, b, x, c.skip);             \
    break;
    EG_BG(4) EG_BG(8) EG_BG(12) EG_BG(16) EG_BG(20) EG_BG(24) EG_BG(28) EG_BG(32) EG_BG(36)
#undef EG_BG
    default:
      block_gemv_kernel<0><<<grid, 256, 0, c.stream>>>(inv, nblocks, bs, b, x, c.skip);
  }
  EG_CUDA(cudaGetLastError());
}

void launch_schur_jacobi(Ctx &c, bool factor) {
  c.ensure_pc_hdg();
  ProfScope ps(c, EG_K_SCHUR_JACOBI, 1);
  const int grid = std::min(c.nf, sm_count_hdg() * 32);
  const int wgrid = std::min((c.nf + 3) / 4, sm_count_hdg() * 32);  // 4 warps (faces) per CTA
  switch (c.t) {
#define EG_SJW(TT)                                                                                     \
  case TT:                                                                                             \
    schur_jacobi_warp_kernel<TT><<<wgrid, 128, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.nf, c.geo.npan, c.D, c.panels, \
                                                              c.pc_hdg, c.piv_hdg, factor, c.derr);      \
    break;
    EG_SJW(4) EG_SJW(8) EG_SJW(12) EG_SJW(16) EG_SJW(20) EG_SJW(24) EG_SJW(28) EG_SJW(32)
#undef EG_SJW
    case 36:
      schur_jacobi_kernel<36><<<grid, 64, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.nf, c.geo.npan, c.D, c.panels, c.pc_hdg,
                                                         c.piv_hdg, factor, c.derr);
      break;
    default:
      fail(EG_ERR_INVALID, "unsupported trace block size");
  }
  EG_CUDA(cudaGetLastError());
}

}  // namespace eg

// Element-wise pivot_reciprocal of n values (host arrays), for the test that
// bounds it against IEEE division.
namespace eg {
namespace {
__global__ void pivot_reciprocal_kernel(long long n, const double *__restrict__ x, double *__restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = pivot_reciprocal(x[i]);
}
}  // namespace
}  // namespace eg

extern "C" int eg_check_pivot_reciprocal(const double *x, double *y, long long n) {
  if (!x || !y || n <= 0) return EG_ERR_INVALID;
  double *d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * 2 * (size_t)n) != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_OUT_OF_MEMORY;
  }
  cudaError_t e = cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    eg::pivot_reciprocal_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 1024), 256>>>(n, d, d + n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(y, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_CUDA;
  }
  return EG_OK;
}
