// Dense direct solve of the assembled Newton system (LinearSolver::Solve with
// --solver dense, src/linear.cpp:46-49, 204-206 and 224-225: the assembled
// CSR converted to a dense matrix, factored by MFEM's DenseMatrixInverse and
// applied to the right-hand side). It serves the reference's small-case
// direct references (at most 5000 unknowns), not the hot path.
//
// The matrix is scattered from the block-sparse full assembly (column-major
// blocks) into a column-major N x N array and factored by right-looking LU
// with partial pivoting as LUFactors::Factor does it: per column the row of
// largest magnitude (first on ties, NaN never chosen) is swapped with the
// pivot row across all columns, the column below the pivot is multiplied by
// the pivot's reciprocal, and the trailing matrix takes the rank-1 update.
// The solve applies the row swaps in order, then the unit-lower and the
// upper triangular sweeps (LUFactors::Solve). A zero pivot is not trapped:
// as in the reference, the non-finite solution fails the caller's residual
// test.
#include <algorithm>

#include "eg_internal.h"

namespace eg {
namespace {

constexpr int kPivThreads = 1024;

__global__ void dense_scatter_kernel(int nnzb, int B, const int *__restrict__ erow, const int *__restrict__ col,
                                     const double *__restrict__ data, int N, double *__restrict__ A) {
  const long long BB = (long long)B * B, total = (long long)nnzb * BB;
  for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(id / BB), e = (int)(id % BB), j = e / B, r = e % B;
    A[(size_t)(col[k] * B + j) * N + (size_t)erow[k] * B + r] = data[id];
  }
}

// Column k: pivot search, row swap over all columns, scaling below the pivot
// (one CTA).
__global__ void __launch_bounds__(kPivThreads) dense_pivot_kernel(int N, int k, double *__restrict__ A,
                                                                  int *__restrict__ piv) {
  __shared__ double sval[kPivThreads];
  __shared__ int sidx[kPivThreads];
  const int t = threadIdx.x;
  double best = 0.;
  int bi = N;  // none yet
  for (int i = k + t; i < N; i += kPivThreads) {
    const double a = fabs(A[(size_t)k * N + i]);
    if (a == a && (bi == N || a > best)) {  // ascending i: strict > keeps the first maximum
      best = a;
      bi = i;
    }
  }
  sval[t] = best;
  sidx[t] = bi;
  __syncthreads();
  for (int s = kPivThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
      const double v = sval[t + s];
      const int ix = sidx[t + s];
      if (ix < N && (sidx[t] == N || v > sval[t] || (v == sval[t] && ix < sidx[t]))) {
        sval[t] = v;
        sidx[t] = ix;
      }
    }
    __syncthreads();
  }
  const int p = sidx[0] < N ? sidx[0] : k;  // an all-NaN column keeps its own row
  if (t == 0) piv[k] = p;
  if (p != k)
    for (int j = t; j < N; j += kPivThreads) {
      double *cj = A + (size_t)j * N;
      const double a = cj[k];
      cj[k] = cj[p];
      cj[p] = a;
    }
  __syncthreads();
  const double inv = 1.0 / A[(size_t)k * N + k];
  for (int i = k + 1 + t; i < N; i += kPivThreads) A[(size_t)k * N + i] *= inv;
}

// Trailing update A[i, j] -= A[i, k] A[k, j], i, j > k (rows contiguous).
__global__ void dense_update_kernel(int N, int k, double *__restrict__ A) {
  const int i = k + 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double lik = A[(size_t)k * N + i];
  for (int j = k + 1 + blockIdx.y; j < N; j += gridDim.y) {
    double *cj = A + (size_t)j * N;
    cj[i] -= lik * cj[k];
  }
}

// x = A^{-1} b with the factors: row swaps in order, L (unit) then U sweeps.
__global__ void __launch_bounds__(kPivThreads) dense_solve_kernel(int N, const double *__restrict__ A,
                                                                  const int *__restrict__ piv,
                                                                  const double *__restrict__ b, double *x) {
  const int t = threadIdx.x;
  for (int i = t; i < N; i += kPivThreads) x[i] = b[i];
  __syncthreads();
  if (t == 0)
    for (int i = 0; i < N; ++i) {
      const int p = piv[i];
      const double a = x[i];
      x[i] = x[p];
      x[p] = a;
    }
  __syncthreads();
  for (int k = 0; k < N; ++k) {
    const double xk = x[k];
    for (int i = k + 1 + t; i < N; i += kPivThreads) x[i] -= A[(size_t)k * N + i] * xk;
    __syncthreads();
  }
  for (int k = N - 1; k >= 0; --k) {
    if (t == 0) x[k] = x[k] / A[(size_t)k * N + k];
    __syncthreads();
    const double xk = x[k];
    for (int i = t; i < k; i += kPivThreads) x[i] -= A[(size_t)k * N + i] * xk;
    __syncthreads();
  }
}

}  // namespace

void dense_factor(Ctx &c, int form) {
  const IluPlan &P = c.ilu[form];
  if (!P.built || !P.asmd) fail(EG_ERR_INVALID, "dense solve requires the full assembly");
  const int N = P.rows * P.B;
  if (N > kDenseMaxUnknowns) fail(EG_ERR_INVALID, "Dense direct solve limited to 5000 unknowns");
  if (c.dense_n != N) {
    c.dense_a = c.alloc_n<double>((size_t)N * N);
    c.dense_piv = c.alloc_n<int>((size_t)N);
    c.dense_n = N;
  }
  ProfScope ps(c, EG_K_VECTOR, 1);
  EG_CUDA(cudaMemsetAsync(c.dense_a, 0, sizeof(double) * (size_t)N * N, c.stream));
  const long long total = (long long)P.nnzb * P.B * P.B;
  const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  dense_scatter_kernel<<<grid, 256, 0, c.stream>>>(P.nnzb, P.B, P.erow, P.col, P.asmd, N, c.dense_a);
  for (int k = 0; k < N; ++k) {
    dense_pivot_kernel<<<1, kPivThreads, 0, c.stream>>>(N, k, c.dense_a, c.dense_piv);
    const int rows = N - k - 1;
    if (rows > 0) {
      const dim3 g((rows + 127) / 128, (unsigned)std::min(rows, 1024));
      dense_update_kernel<<<g, 128, 0, c.stream>>>(N, k, c.dense_a);
    }
  }
  EG_CUDA(cudaGetLastError());
}

void dense_solve(Ctx &c, const double *b, double *x) {
  if (!c.dense_a) fail(EG_ERR_INVALID, "dense solve before its factorization");
  ProfScope ps(c, EG_K_VECTOR, 1);
  dense_solve_kernel<<<1, kPivThreads, 0, c.stream>>>(c.dense_n, c.dense_a, c.dense_piv, b, x);
  EG_CUDA(cudaGetLastError());
}

}  // namespace eg
