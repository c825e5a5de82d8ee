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
template <int Q>
__global__ void __launch_bounds__(256)
    condense_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                    const double *__restrict__ r, double *XY, double *Cb, double *sf_out,
                    double *contrib, double *panels, double *work, int *err) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
  constexpr int MODE = condense_mode<Q>();
  __shared__ STab<Q> st;
  __shared__ double us[M], UT[16 * Q], FM[4 * Q * 16], SF[4 * Q], CB[4 * Q * 16];
  __shared__ int piv_s[M];
  __shared__ double inv_piv[M];
  __shared__ double bcast[2];
  extern __shared__ double dyn[];
  load_tables<Q>(st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += blockDim.x) us[i] = u[(size_t)e * M + i];
    __syncthreads();
    for (int task = threadIdx.x; task < 4 * Q; task += blockDim.x) {
      const int s = task / Q, j = task % Q;
      double o[4] = {0., 0., 0., 0.};
      for (int l = 0; l < Q; ++l) {
        const double f = st.fb(s, j, l);
        const double *v = us + 4 * line_node<Q>(s, j, l);
#pragma unroll
        for (int c = 0; c < 4; ++c) o[c] += f * v[c];
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) UT[task * 4 + c] = o[c];
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
      jacobian(UT + 4 * task, s < 2 ? 0 : 1, g.gm1, jm);
      const double nsign = L ? 1. : -1.;
      const double ewj = st.ew(j);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const double v = nsign * jm[k] + ((k % 5) == 0 ? stab : 0.);
        FM[task * 16 + k] = v;
        const double cv = -ewj * v;
        CB[task * 16 + k] = cv;
        Cb[((size_t)e * 4 * Q + task) * 16 + k] = cv;
      }
      const double len = s < 2 ? g.hy : g.hx;
      const double scale = g.dt * len / g.area * ewj;
      const double sv = -scale * stab;
      SF[task] = sv;
      sf_out[(size_t)e * 4 * Q + task] = sv;
    }
    __syncthreads();
    double *A = MODE < 2 ? dyn : work + (size_t)blockIdx.x * M * M;
    double *R = MODE == 0 ? dyn + (size_t)M * M : XY + (size_t)e * M * NR;
    build_cell_matrix<Q>(A, M, st, us, FM, g);
    for (int col = threadIdx.x; col < NR; col += blockDim.x) {
      double *rc = R + (size_t)col * M;
      if (col < 4 * T) {
        for (int i = 0; i < M; ++i) rc[i] = 0.;
        const int s = col / T, jj = (col % T) >> 2, c = col & 3;
        const double sv = SF[s * Q + jj];
        for (int l = 0; l < Q; ++l) {
          const int i = line_node<Q>(s, jj, l);
          rc[4 * i + c] = st.fb(s, jj, l) * st.inv_mass(i) * sv;
        }
      } else {
        for (int i = 0; i < M; ++i) rc[i] = r[(size_t)e * M + i];
      }
    }
    __syncthreads();
    const bool ok = cta_lu_solve<(M + 31) / 32>(A, M, R, M, M, NR, piv_s, inv_piv, bcast);
    if (!ok) {
      if (threadIdx.x == 0) raise_err(err, DERR_SINGULAR_CELL);
      continue;
    }
    if (MODE == 0) {
      double *dst = XY + (size_t)e * M * NR;
      for (int i = threadIdx.x; i < M * NR; i += blockDim.x) dst[i] = R[i];
    }
    // rhs contributions C_e y_e (src/condensation.cpp:141-142)
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
      const double *cb = CB + (s * Q + jj) * 16;
      double res = 0.;
#pragma unroll
      for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * val[d];
      contrib[(size_t)e * 4 * T + o] = res;
    }
    // Schur Jacobi panels C_s X_s (src/operators.cpp:7-26, 295-301)
    if (panels) {
      for (int o = threadIdx.x; o < 4 * T * T; o += blockDim.x) {
        const int s = o / (T * T), rem = o % (T * T);
        const int row = rem % T, cc = rem / T;
        const int jj = row >> 2, c = row & 3;
        const double *xc = R + (size_t)(s * T + cc) * M;
        double val[4] = {0., 0., 0., 0.};
        for (int l = 0; l < Q; ++l) {
          const double f = st.fb(s, jj, l);
          const double *xv = xc + 4 * line_node<Q>(s, jj, l);
#pragma unroll
          for (int d = 0; d < 4; ++d) val[d] += f * xv[d];
        }
        const double *cb = CB + (s * Q + jj) * 16;
        double res = 0.;
#pragma unroll
        for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * val[d];
        panels[(size_t)e * 4 * T * T + o] = res;
      }
    }
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
                     double *__restrict__ out) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1;
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

// y_f = D_f v_f - contrib[L][ls] - contrib[R][rs]  (one thread per trace dof)
__global__ void face_combine_kernel(int nx, int ny, int T, int nl, const double *__restrict__ D,
                                    const double *__restrict__ v, const double *__restrict__ contrib,
                                    double sign_v, double *__restrict__ y) {
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

// Schur block-Jacobi: S_ff = D_f - P_L - P_R, then pivoted LU in place
// (ElementOperator::DiagonalBlocks src/operators.cpp:275-303 + linear.cpp:198-202).
template <int T>
__global__ void __launch_bounds__(64)
    schur_jacobi_kernel(int nx, int ny, int nf, const double *__restrict__ D,
                        const double *__restrict__ panels, double *blocks, int *pivots, bool factor,
                        int *err) {
  __shared__ double S[T * T];
  __shared__ int piv_s[T];
  __shared__ double inv_piv[T];
  __shared__ double bcast[2];
  for (int f = blockIdx.x; f < nf; f += gridDim.x) {
    __syncthreads();
    const int L = f >> 1, ls = (f & 1) ? 3 : 1;
    const int R = neighbour(L, ls, nx, ny), rs = ls - 1;
    const double *pl = panels + ((size_t)L * 4 + ls) * T * T;
    const double *pr = panels + ((size_t)R * 4 + rs) * T * T;
    for (int o = threadIdx.x; o < T * T; o += blockDim.x) {
      const int row = o % T, col = o / T;
      const double d = row == col ? D[(size_t)f * T + row] : 0.;
      S[o] = (d - pl[o]) - pr[o];
    }
    __syncthreads();
    if (factor) {
      const bool ok = cta_lu_solve<(T + 31) / 32>(S, T, nullptr, 1, T, 0, piv_s, inv_piv, bcast);
      if (!ok && threadIdx.x == 0) raise_err(err, DERR_SINGULAR_JACOBI);
    } else {
      for (int i = threadIdx.x; i < T; i += blockDim.x) piv_s[i] = i;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < T * T; o += blockDim.x) blocks[(size_t)f * T * T + o] = S[o];
    for (int i = threadIdx.x; i < T; i += blockDim.x) pivots[(size_t)f * T + i] = piv_s[i];
  }
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

void launch_condense(Ctx &c, const double *u, const double *r) {
  c.ensure_hdg();
  const int grid = condense_grid(c);
  ProfScope ps(c, EG_K_CONDENSE, 2);
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
  EG_CUDA(cudaGetLastError());
  // rhs_f = contrib_L + contrib_R (s.rhs = 0; rhs[ids] += C y)
  const int blocks = (c.nl + 255) / 256;
  face_combine_kernel<<<blocks, 256, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.t, c.nl, nullptr, c.rhs,
                                                    c.contrib, -1.0, c.rhs);
  EG_CUDA(cudaGetLastError());
  c.condensed = true;
}

void launch_schur_apply(Ctx &c, const double *v, double *y) {
  ProfScope ps(c, EG_K_SCHUR_APPLY, 2);
  const int grid = std::min(c.n, sm_count_hdg() * 16);
  EG_DISPATCH_Q(c.q, (cell_gemv_kernel<Q, false><<<grid, 128, 0, c.stream>>>(c.geo, c.tab, c.XY, c.Cb,
                                                                            v, c.contrib)));
  EG_CUDA(cudaGetLastError());
  const int blocks = (c.nl + 255) / 256;
  face_combine_kernel<<<blocks, 256, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.t, c.nl, c.D, v,
                                                    c.contrib, 1.0, y);
  EG_CUDA(cudaGetLastError());
}

void launch_recover(Ctx &c, const double *lam, double *du) {
  ProfScope ps(c, EG_K_RECOVER, 1);
  const int grid = std::min(c.n, sm_count_hdg() * 16);
  EG_DISPATCH_Q(c.q, (cell_gemv_kernel<Q, true><<<grid, 128, 0, c.stream>>>(c.geo, c.tab, c.XY, c.Cb,
                                                                           lam, du)));
  EG_CUDA(cudaGetLastError());
}

void launch_recovered_residual(Ctx &c, const double *eq, double *er) {
  const int total = c.n * c.p;
  ProfScope ps(c, EG_K_RECOVERED_RESIDUAL, 1);
  EG_DISPATCH_Q(c.q, (recovered_residual_kernel<Q><<<(total + 255) / 256, 256, 0, c.stream>>>(
                         c.geo, c.tab, c.sf, c.D, eq, er)));
  EG_CUDA(cudaGetLastError());
}

void launch_schur_jacobi(Ctx &c, bool factor) {
  c.ensure_pc_hdg();
  ProfScope ps(c, EG_K_SCHUR_JACOBI, 1);
  const int grid = std::min(c.nf, sm_count_hdg() * 32);
  switch (c.t) {
#define EG_SJ(TT)                                                                                 \
  case TT:                                                                                        \
    schur_jacobi_kernel<TT><<<grid, 64, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.nf, c.D, c.panels, \
                                                       c.pc_hdg, c.piv_hdg, factor, c.derr);             \
    break;
    EG_SJ(4) EG_SJ(8) EG_SJ(12) EG_SJ(16) EG_SJ(20) EG_SJ(24) EG_SJ(28) EG_SJ(32) EG_SJ(36)
#undef EG_SJ
    default:
      fail(EG_ERR_INVALID, "unsupported trace block size");
  }
  EG_CUDA(cudaGetLastError());
}

}  // namespace eg
