// Mixed precision for the condensed HDG solve: FP64 iterative refinement of
// S lambda = rhs around an FP32 inner GMRES.
//
// What stays FP64: the residual, the HLL bounds, the condensation (X, y), the
// outer residual rhs - S lambda with the FP64 X, the correction update of
// lambda, the recovery du = -X lambda - y and the Newton/line-search tests.
// What runs in FP32: a copy of X for the inner Schur action, the Schur
// block-Jacobi inverses (factored in FP64, stored in FP32) and the inner
// Krylov vectors; their dot products and the Hessenberg/Givens work stay FP64.
// Each refinement step scales the current FP64 residual to unit norm, solves
// the FP32 system to a relative tolerance of kInnerTol (or looser when less
// is needed to reach the outer target), and adds the correction in FP64.
// The outer loop stops at the same relative residual as the FP64 solver
// (LinearSolver::Impl::GMRES, src/linear.cpp:76-157), so the Newton update
// meets the reference's acceptance tests unchanged.
#include <algorithm>
#include <cmath>

#include "eg_internal.h"

namespace eg {
namespace {

constexpr double kInnerTol = 1e-5;
constexpr int kMaxRefine = 40;

int vgrid(long long n) { return (int)std::max(1LL, std::min((n + 255) / 256, 148LL * 16)); }

__global__ void to_f32_kernel(long long n, const double *__restrict__ x, float *__restrict__ y) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// X part of every cell's [X | y] (m x (4t+1), column-major) into an m x 4t
// FP32 block.
__global__ void x_to_f32_kernel(long long n_cells, int M, int NR, const double *__restrict__ XY,
                                float *__restrict__ Xf) {
  const long long per = (long long)M * (NR - 1), total = n_cells * per;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long e = i / per, o = i % per;
    Xf[i] = (float)XY[e * (long long)M * NR + o];
  }
}

// rf = r / |r|, rounded to FP32
__global__ void scaled_to_f32_kernel(int n, double s, const double *__restrict__ r, float *__restrict__ rf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rf[i] = (float)(r[i] * s);
}
// x += a * d  (FP64 accumulation of an FP32 correction)
__global__ void add_scaled_f32_kernel(int n, double a, const float *__restrict__ d, double *__restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += a * (double)d[i];
}

// FP32 Schur action, cell part: contrib_e = C_e R (X_e v_e) (the FP32 twin of
// the FP64 cell GEMV of ElementOperator::Mult, src/operators.cpp:166-178).
template <int Q>
__global__ void __launch_bounds__(128)
    cell_gemv_f32_kernel(Geo g, const double *__restrict__ tab, const float *__restrict__ Xf,
                         const double *__restrict__ Cb, const float *__restrict__ v, float *__restrict__ out,
                         const int *__restrict__ skip) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q;
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  __shared__ STab<Q> st;
  __shared__ float vl[4 * T], mid[M];
  load_tables<Q>(st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * T; i += blockDim.x) {
      const int s = i / T;
      vl[i] = v[(size_t)cell_face(e, s, g.nx, g.ny) * T + (i % T)];
    }
    __syncthreads();
    const float *X = Xf + (size_t)e * M * 4 * T;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
      float acc = 0.f;
#pragma unroll 8
      for (int col = 0; col < 4 * T; ++col) acc = fmaf(X[(size_t)col * M + i], vl[col], acc);
      mid[i] = acc;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < 4 * T; o += blockDim.x) {
      const int s = o / T, jj = (o % T) >> 2, c = o & 3;
      float val[4] = {0.f, 0.f, 0.f, 0.f};
      for (int l = 0; l < Q; ++l) {
        const float f = (float)st.fb(s, jj, l);
        const float *mv = mid + 4 * line_node<Q>(s, jj, l);
#pragma unroll
        for (int d = 0; d < 4; ++d) val[d] += f * mv[d];
      }
      const double *cb = Cb + ((size_t)e * 4 * Q + s * Q + jj) * 16;
      float res = 0.f;
#pragma unroll
      for (int d = 0; d < 4; ++d) res += (float)cb[c + 4 * d] * val[d];
      out[(size_t)e * 4 * T + o] = res;
    }
  }
}

// FP32 Schur action from FP32 copies of the 16 panels C_s X_o of a cell
// (wherever all 16 panels are kept; the FP64 panel form is panel_gemv_kernel).
template <int Q>
__global__ void __launch_bounds__(((16 * Q + 31) / 32) * 32)
    panel_gemv_f32_kernel(Geo g, const float *__restrict__ panels, const float *__restrict__ v,
                          float *__restrict__ out, const int *__restrict__ skip) {
  constexpr int T = 4 * Q, TT = T * T;
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  __shared__ float vl[4 * T];
  const int o = threadIdx.x, s = o / T, row = o % T;
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * T; i += blockDim.x)
      vl[i] = v[(size_t)cell_face(e, i / T, g.nx, g.ny) * T + (i % T)];
    __syncthreads();
    if (o < 4 * T) {
      const float *P = panels + ((size_t)e * 16 + s * 4) * TT + row;
      float acc = 0.f;
#pragma unroll 8
      for (int k = 0; k < 4 * T; ++k) acc = fmaf(P[(size_t)(k / T) * TT + (k % T) * T], vl[k], acc);
      out[(size_t)e * 4 * T + o] = acc;
    }
  }
}

// y_f = D_f v_f - contrib[L][ls] - contrib[R][rs]
__global__ void face_combine_f32_kernel(int nx, int ny, int T, int nl, const float *__restrict__ D,
                                        const float *__restrict__ v, const float *__restrict__ contrib,
                                        float *__restrict__ y, const int *__restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nl) return;
  const int f = idx / T, i = idx % T;
  const int L = f >> 1, ls = (f & 1) ? 3 : 1;
  const int R = neighbour(L, ls, nx, ny), rs = ls - 1;
  y[idx] = (D[idx] * v[idx] - contrib[(size_t)L * 4 * T + ls * T + i]) - contrib[(size_t)R * 4 * T + rs * T + i];
}

// x_b = Inv_b b_b for row-major FP32 block inverses; one thread per row (BS > 0:
// compile-time block size, the row loop unrolls; BS = 0: any multiple of 4).
template <int BS>
__global__ void __launch_bounds__(256)
    block_gemv_f32_kernel(const float *__restrict__ inv, int nblocks, int bs_rt, const float *__restrict__ b,
                          float *__restrict__ x, const int *__restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int bs = BS > 0 ? BS : bs_rt;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (long long)nblocks * bs) return;
  const int blk = (int)(id / bs);
  const float4 *ib = reinterpret_cast<const float4 *>(inv + (size_t)id * bs);  // row-major, bs % 4 == 0
  const float *bb = b + (size_t)blk * bs;
  float acc = 0.f;
#pragma unroll
  for (int c = 0; c < (BS > 0 ? BS / 4 : bs / 4); ++c) {
    const float4 a = ib[c];
    acc = fmaf(a.x, bb[4 * c], acc);
    acc = fmaf(a.y, bb[4 * c + 1], acc);
    acc = fmaf(a.z, bb[4 * c + 2], acc);
    acc = fmaf(a.w, bb[4 * c + 3], acc);
  }
  x[id] = acc;
}

int sm_count_mixed() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Inner operators: FP32 Schur action and FP32 block-Jacobi apply.
struct MixedHdgOps : LinearOpsT<float> {
  explicit MixedHdgOps(Ctx &c) {
    N = c.nl;
    mtab = c.mtab_hdg;
    period = 2 * c.t;
    group = kArnoldiGroup;
  }
  void apply(Ctx &c, const float *x, float *y) override {
    ProfScope ps(c, EG_K_SCHUR_APPLY, 2);
    const int grid = std::min(c.n, sm_count_mixed() * 16);
    if (c.geo.npan == 16) {  // Xf holds the FP32 panels
      switch (c.q) {
#define EG_PGF(QQ)                                                                                    \
  case QQ:                                                                                            \
    panel_gemv_f32_kernel<QQ><<<grid, ((16 * QQ + 31) / 32) * 32, 0, c.stream>>>(c.geo, c.Xf, x, c.contribf, \
                                                                                c.skip);              \
    break;
        EG_PGF(1) EG_PGF(2) EG_PGF(3) EG_PGF(4) EG_PGF(5) EG_PGF(6) EG_PGF(7) EG_PGF(8) EG_PGF(9)
#undef EG_PGF
        default:
          fail(EG_ERR_INVALID, "unsupported degree");
      }
    } else {
      EG_DISPATCH_Q(c.q, (cell_gemv_f32_kernel<Q><<<grid, 128, 0, c.stream>>>(c.geo, c.tab, c.Xf, c.Cb, x,
                                                                            c.contribf, c.skip)));
    }
    EG_CUDA(cudaGetLastError());
    face_combine_f32_kernel<<<(c.nl + 255) / 256, 256, 0, c.stream>>>(c.desc.nx, c.desc.ny, c.t, c.nl, c.Df, x,
                                                                      c.contribf, y, c.skip);
    EG_CUDA(cudaGetLastError());
  }
  void precondition(Ctx &c, const float *b, float *x) override {
    ProfScope ps(c, EG_K_PC_APPLY, 1);
    const long long total = (long long)c.nf * c.t;
    const unsigned grid = (unsigned)((total + 255) / 256);
    switch (c.t) {
#define EG_BGF(BB)                                                                              \
  case BB:                                                                                      \
    block_gemv_f32_kernel<BB><<<grid, 256, 0, c.stream>>>(c.pcf, c.nf, c.t, b, x, c.skip);       \
    break;
      EG_BGF(4) EG_BGF(8) EG_BGF(12) EG_BGF(16) EG_BGF(20) EG_BGF(24) EG_BGF(28) EG_BGF(32) EG_BGF(36)
#undef EG_BGF
      default:
        block_gemv_f32_kernel<0><<<grid, 256, 0, c.stream>>>(c.pcf, c.nf, c.t, b, x, c.skip);
    }
    EG_CUDA(cudaGetLastError());
  }
};

void ensure_mixed(Ctx &c) {
  if (c.Xf) return;
  c.ensure_krylov();  // fixes the restart length both solvers use
  // FP32 copy of X, or of the 16 Schur panels per cell where the FP64 Schur
  // action streams those (all 16 panels kept per cell)
  c.Xf = c.alloc_n<float>((size_t)c.n * (c.geo.npan == 16 ? 16 * c.t * c.t : c.m * 4 * c.t));
  c.pcf = c.alloc_n<float>((size_t)c.nf * c.t * c.t);
  c.Df = c.alloc_n<float>(c.nl);
  c.contribf = c.alloc_n<float>((size_t)c.n * 4 * c.t);
  const size_t N = c.nl;
  c.kfV = c.alloc_n<float>(N * (c.kR + 1));
  c.kfw = c.alloc_n<float>(N);
  c.kfz = c.alloc_n<float>(N);
  c.kfres = c.alloc_n<float>(N);
  c.kfcomb = c.alloc_n<float>(N);
  c.kfcorr = c.alloc_n<float>(N);
  c.kfx = c.alloc_n<float>(N);
  c.kfrhs = c.alloc_n<float>(N);
}

}  // namespace

void mixed_prepare(Ctx &c) {
  ensure_mixed(c);
  ProfScope ps(c, EG_K_VECTOR, 3);
  if (c.geo.npan == 16) {
    const long long npan = (long long)c.n * 16 * c.t * c.t;
    to_f32_kernel<<<vgrid(npan), 256, 0, c.stream>>>(npan, c.panels, c.Xf);
  } else {
    const long long nx = (long long)c.n * c.m * 4 * c.t;
    x_to_f32_kernel<<<vgrid(nx), 256, 0, c.stream>>>(c.n, c.m, 4 * c.t + 1, c.XY, c.Xf);
  }
  const long long np = (long long)c.nf * c.t * c.t;
  to_f32_kernel<<<vgrid(np), 256, 0, c.stream>>>(np, c.pc_hdg, c.pcf);
  to_f32_kernel<<<vgrid(c.nl), 256, 0, c.stream>>>(c.nl, c.D, c.Df);
  EG_CUDA(cudaGetLastError());
}

double schur_refine_mixed(Ctx &c, const double *rhs, double *x, bool zero_guess, double tol, int limit,
                          double rhs_norm, int *count) {
  c.ensure_krylov();
  ensure_mixed(c);
  const int N = c.nl;
  double *res = c.kres, *tmp = c.kw;
  if (zero_guess) {
    launch_fill(c, N, 0., x);
    launch_copy(c, N, rhs, res);
  } else {
    launch_schur_apply(c, x, tmp);
    launch_axpby(c, N, 1., rhs, -1., tmp, res);
  }
  double rn = wnorm(c, res, N, c.mtab_hdg, 2 * c.t);
  MixedHdgOps ops(c);
  const KrylovBufs<float> kb{c.kfV, c.kfw, c.kfz, c.kfres, c.kfcomb, c.kfcorr, (size_t)N, c.kR};
  int total = 0;
  for (int outer = 0; outer < kMaxRefine && rn > tol * rhs_norm && total < limit; ++outer) {
    scaled_to_f32_kernel<<<vgrid(N), 256, 0, c.stream>>>(N, 1. / rn, res, c.kfrhs);
    EG_CUDA(cudaGetLastError());
    const double inner_tol = std::max(kInnerTol, 0.1 * tol * rhs_norm / rn);
    int cnt = 0;
    gmres_f32(c, ops, kb, c.kfrhs, c.kfx, inner_tol, limit - total, &cnt);
    total += cnt;
    {
      ProfScope ps(c, EG_K_VECTOR, 1);
      add_scaled_f32_kernel<<<vgrid(N), 256, 0, c.stream>>>(N, rn, c.kfx, x);
      EG_CUDA(cudaGetLastError());
    }
    launch_schur_apply(c, x, tmp);
    launch_axpby(c, N, 1., rhs, -1., tmp, res);
    const double next = wnorm(c, res, N, c.mtab_hdg, 2 * c.t);
    if (!std::isfinite(next)) fail(EG_ERR_GMRES_NONFINITE, "Nonfinite GMRES residual");
    const bool stalled = cnt == 0 || !(next < rn);
    rn = next;
    if (stalled) break;
  }
  *count = total;
  if (!(rn <= tol * rhs_norm)) fail(EG_ERR_GMRES_LIMIT, "GMRES iteration limit reached");
  return rn;
}

}  // namespace eg
