// Device-side building blocks shared by all kernels: the ideal-gas physics,
// periodic Cartesian topology, shared-memory table staging and the
// CTA-cooperative pivoted LU used by condensation and block Jacobi.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace eg {

// ----------------------------------------------------------------- geometry
// Scalar description of one instance (passed by value to kernels).
struct Geo {
  int nx, ny, n, nf;
  double hx, hy, area, dt, gamma, gm1, safety;
  int npan;  // Schur panels C_s X_o stored per cell: the 4 diagonal ones or all 16
};

// Frozen per-face-point HLL data (src/problem.cpp:357-374), SoA of nf*q.
struct Frozen {
  const double *a, *b, *lw, *rw, *pen;
};

// Flat per-instance table block in global memory; offsets for a given Q.
// [tdx Q*Q][tdy Q*Q][fb 4*Q*Q][w Q*Q][inv_mass Q*Q][mass Q*Q][ew Q]
template <int Q>
struct TabLayout {
  static constexpr int P = Q * Q;
  static constexpr int TDX = 0, TDY = P, FB = 2 * P, W = 6 * P, IM = 7 * P, MS = 8 * P, EW = 9 * P;
  static constexpr int SIZE = 9 * P + Q;
};
__host__ __device__ constexpr int tab_size(int q) { return 9 * q * q + q; }

template <int Q>
struct STab {
  double d[TabLayout<Q>::SIZE];
  __device__ __forceinline__ double tdx(int a, int i) const { return d[TabLayout<Q>::TDX + a * Q + i]; }
  __device__ __forceinline__ double tdy(int a, int j) const { return d[TabLayout<Q>::TDY + a * Q + j]; }
  // face_basis value of normal-line node l for side s, face point j
  __device__ __forceinline__ double fb(int s, int j, int l) const {
    return d[TabLayout<Q>::FB + (s * Q + j) * Q + l];
  }
  __device__ __forceinline__ double w(int i) const { return d[TabLayout<Q>::W + i]; }
  __device__ __forceinline__ double inv_mass(int i) const { return d[TabLayout<Q>::IM + i]; }
  __device__ __forceinline__ double mass(int i) const { return d[TabLayout<Q>::MS + i]; }
  __device__ __forceinline__ double ew(int j) const { return d[TabLayout<Q>::EW + j]; }
};

template <int Q>
__device__ __forceinline__ void load_tables(STab<Q> &st, const double *__restrict__ tab) {
  for (int i = threadIdx.x; i < TabLayout<Q>::SIZE; i += blockDim.x) st.d[i] = tab[i];
}

// Native node index of normal-line node l through face point j of side s.
template <int Q>
__device__ __forceinline__ int line_node(int s, int j, int l) {
  return s < 2 ? j * Q + l : l * Q + j;
}

// Periodic neighbours; sides 0=x-, 1=x+, 2=y-, 3=y+ (src/problem.cpp:150-156).
__host__ __device__ __forceinline__ int neighbour(int e, int s, int nx, int ny) {
  const int ix = e % nx, iy = e / nx;
  switch (s) {
    case 0: return iy * nx + (ix == 0 ? nx - 1 : ix - 1);
    case 1: return iy * nx + (ix == nx - 1 ? 0 : ix + 1);
    case 2: return (iy == 0 ? ny - 1 : iy - 1) * nx + ix;
    default: return (iy == ny - 1 ? 0 : iy + 1) * nx + ix;
  }
}
// Face of cell e on side s; the cell is the face's left cell on sides 1 and 3.
__host__ __device__ __forceinline__ int cell_face(int e, int s, int nx, int ny) {
  if (s == 1) return 2 * e;
  if (s == 3) return 2 * e + 1;
  return 2 * neighbour(e, s, nx, ny) + (s == 2 ? 1 : 0);
}
__device__ __forceinline__ bool side_is_left(int s) { return s == 1 || s == 3; }

// Trace of the 4 components of cell c at side s, face point j (Problem::Eval
// with fv[side], src/problem.cpp:244-250).
template <int Q>
__device__ __forceinline__ void trace4(const STab<Q> &st, const double *__restrict__ u, int c,
                                       int s, int j, double out[4]) {
  out[0] = out[1] = out[2] = out[3] = 0.;
  const double *cell = u + (size_t)c * (4 * Q * Q);
#pragma unroll
  for (int l = 0; l < Q; ++l) {
    const double f = st.fb(s, j, l);
    const double *v = cell + 4 * line_node<Q>(s, j, l);
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] += f * v[k];
  }
}

// ------------------------------------------------------------------ physics
// Restates EulerGas (src/physics.cpp:5-63). State order (rho, rho vx, rho vy, E).
__device__ __forceinline__ double pressure(const double u[4], double gm1) {
  return gm1 * (u[3] - .5 * (u[1] * u[1] + u[2] * u[2]) / u[0]);
}
__device__ __forceinline__ bool positive(const double u[4], double gm1) {
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (!isfinite(u[c])) return false;
  return u[0] > 1e-13 && pressure(u, gm1) > 1e-13;
}
__device__ __forceinline__ void flux(const double u[4], int axis, double gm1, double f[4]) {
  const double vn = u[axis + 1] / u[0], p = pressure(u, gm1);
  f[0] = u[axis + 1];
  f[1] = u[1] * vn;
  f[2] = u[2] * vn;
  f[3] = (u[3] + p) * vn;
  f[axis + 1] += p;
}
// Column-major 4x4 flux Jacobian j[c + 4 d] = dF_c/dU_d.
__device__ __forceinline__ void jacobian(const double u[4], int axis, double gm1, double j[16]) {
  const double inv = 1. / u[0];
  const double vx = u[1] * inv, vy = u[2] * inv;
  const double vn = u[axis + 1] * inv;
  const double hd = u[3] + pressure(u, gm1);
  const double dp[4] = {.5 * gm1 * (vx * vx + vy * vy), -gm1 * vx, -gm1 * vy, gm1};
  double dv[4] = {-vn * inv, 0., 0., 0.};
  dv[axis + 1] = inv;
#pragma unroll
  for (int c = 0; c < 4; ++c) j[4 * c] = 0.;
  j[4 * (axis + 1)] = 1.;
#pragma unroll
  for (int d = 0; d < 2; ++d) {
#pragma unroll
    for (int c = 0; c < 4; ++c) j[(d + 1) + 4 * c] = u[d + 1] * dv[c] + (axis == d ? dp[c] : 0.);
    j[(d + 1) + 4 * (d + 1)] += vn;
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) j[3 + 4 * c] = vn * dp[c] + hd * dv[c];
  j[3 + 4 * 3] += vn;
}
// y = J x
__device__ __forceinline__ void mat4_vec(const double j[16], const double x[4], double y[4]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) y[c] = 0.;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
#pragma unroll
    for (int c = 0; c < 4; ++c) y[c] += j[c + 4 * d] * x[d];
  }
}

enum DevErr : int {
  DERR_NONE = 0,
  DERR_NONPOSITIVE_FACE = 3,
  DERR_ROE_SOUND = 4,
  DERR_DEGENERATE_HLL = 5,
  DERR_INADMISSIBLE = 6,
  DERR_SINGULAR_CELL = 7,
  DERR_SINGULAR_JACOBI = 8,
  DERR_SINGULAR_ILU = 9,
  DERR_WAIT_LIMIT = 24,
};
__device__ __forceinline__ void raise_err(int *err, int code) { atomicCAS(err, 0, code); }

// Einfeldt/Roe HLL bounds x safety (src/physics.cpp:40-63); returns an error
// code instead of throwing.
__device__ __forceinline__ int hll_speeds(const double l[4], const double r[4], int axis, double gamma,
                                          double gm1, double safety, double &a, double &b) {
  bool finite = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) finite = finite && isfinite(l[c]) && isfinite(r[c]);
  if (!(finite && l[0] > 1e-13 && r[0] > 1e-13)) return DERR_NONPOSITIVE_FACE;
  const double pl = pressure(l, gm1), pr = pressure(r, gm1);
  if (!(pl > 1e-13 && pr > 1e-13)) return DERR_NONPOSITIVE_FACE;
  const double il = 1. / l[0], ir = 1. / r[0];
  const double sl = sqrt(l[0]), sr = sqrt(r[0]);
  double v[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) v[d] = (sl * l[d + 1] * il + sr * r[d + 1] * ir) / (sl + sr);
  const double h = (sl * (l[3] + pl) * il + sr * (r[3] + pr) * ir) / (sl + sr);
  const double c2 = gm1 * (h - .5 * (v[0] * v[0] + v[1] * v[1]));
  if (!(c2 > 0)) return DERR_ROE_SOUND;
  const double ct = sqrt(c2), cl = sqrt(gamma * pl * il), cr = sqrt(gamma * pr * ir);
  a = safety * fmax(0., fmax(cl - l[axis + 1] * il, ct - v[axis]));
  b = safety * fmax(0., fmax(cr + r[axis + 1] * ir, ct + v[axis]));
  return DERR_NONE;
}

// ------------------------------------------------------ CTA pivoted dense LU
// Factor the m x m column-major matrix A (leading dimension lda) in place with
// row partial pivoting (largest magnitude, first index on ties: the order of
// MFEM LUFactors::Factor and LAPACK getf2), applying the same row operations
// to the nb columns of B (leading dimension ldb), then overwrite B with
// A^{-1} B by back substitution (x_j = b_j / u_jj; b_i -= u_ij x_j).
// On exit A holds unit-lower L (below) and U (on/above the diagonal) in the
// packed LAPACK layout and piv[j] is the row exchanged with j at step j.
//
// Row exchanges of a step are applied immediately to the trailing columns;
// the pivot column itself and the finished L columns are exchanged (and the
// L multipliers scaled) in one fix-up pass at the end, so a step needs two CTA
// barriers. RMAX bounds ceil(m/32). A and B may live in shared or global
// memory. Returns false, uniformly across the CTA, on a zero pivot.
template <int RMAX>
__device__ bool cta_lu_solve(double *A, int lda, double *B, int ldb, int m, int nb, int *piv,
                             double *inv_piv, volatile double *bcast) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int ncols = m + nb;
  for (int j = 0; j < m; ++j) {
    if (warp == 0) {
      // largest magnitude, first row on ties, NaN never chosen: magnitudes
      // compared as IEEE bit patterns (integer compares, warp reductions)
      constexpr unsigned long long kAbs = 0x7fffffffffffffffull, kInf = 0x7ff0000000000000ull;
      unsigned long long best = 0ull;
      int bi = m;
      for (int i = j + lane; i < m; i += 32) {
        const unsigned long long bits = (unsigned long long)__double_as_longlong(A[i + (size_t)j * lda]) & kAbs;
        if (bits <= kInf && (bi == m || bits > best)) {
          best = bits;
          bi = i;
        }
      }
      const unsigned hi = (unsigned)(best >> 32), lo = (unsigned)best;
      const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
      const bool c1 = bi < m && hi == mhi;
      const unsigned mlo = __reduce_max_sync(0xffffffffu, c1 ? lo : 0u);
      bi = (int)__reduce_min_sync(0xffffffffu, c1 && lo == mlo ? (unsigned)bi : (unsigned)m);
      if (lane == 0) {
        // an all-NaN column leaves bi == m: report it as a zero pivot
        const double pv = bi < m ? A[bi + (size_t)j * lda] : 0.;
        piv[j] = bi < m ? bi : j;
        bcast[0] = pv;
        const double ip = 1.0 / pv;
        bcast[1] = ip;
        inv_piv[j] = ip;
      }
    }
    __syncthreads();
    const int p = piv[j];
    const double pv = bcast[0];
    if (!(fabs(pv) > 0.)) return false;
    const double inv = bcast[1];
    // multipliers of this lane's rows (virtual exchange of rows j and p)
    double lm[RMAX];
#pragma unroll
    for (int k = 0; k < RMAX; ++k) {
      const int i = j + 1 + lane + 32 * k;
      double v = 0.;
      if (i < m) v = (i == p ? A[j + (size_t)j * lda] : A[i + (size_t)j * lda]) * inv;
      lm[k] = v;
    }
    // two of this warp's columns per iteration (the same columns per warp as
    // one at a time): their reads overlap and share one warp sync
    for (int l0 = j + 1 + warp; l0 < ncols; l0 += 2 * nwarps) {
      const int l1 = l0 + nwarps;
      const bool two = l1 < ncols;
      double *c0 = l0 < m ? A + (size_t)l0 * lda : B + (size_t)(l0 - m) * ldb;
      double *c1 = !two ? c0 : (l1 < m ? A + (size_t)l1 * lda : B + (size_t)(l1 - m) * ldb);
      const double top0 = c0[p], old0 = c0[j];  // values moving to rows j and p
      const double top1 = c1[p], old1 = c1[j];
      __syncwarp();
#pragma unroll
      for (int k = 0; k < RMAX; ++k) {
        const int i = j + 1 + lane + 32 * k;
        if (i < m) {
          const double cur0 = (i == p) ? old0 : c0[i];
          const double cur1 = (i == p) ? old1 : c1[i];
          c0[i] = cur0 - lm[k] * top0;
          if (two) c1[i] = cur1 - lm[k] * top1;
        }
      }
      if (lane == 0) {
        c0[j] = top0;
        if (two) c1[j] = top1;
      }
      __syncwarp();
    }
    __syncthreads();
  }
  // fix-up: deferred exchanges and multiplier scaling of the L columns
  for (int c = threadIdx.x; c < m; c += blockDim.x) {
    double *col = A + (size_t)c * lda;
    for (int j = c; j < m; ++j) {
      const int p = piv[j];
      if (p != j) {
        const double t = col[j];
        col[j] = col[p];
        col[p] = t;
      }
    }
    const double s = inv_piv[c];
    for (int i = c + 1; i < m; ++i) col[i] *= s;
  }
  __syncthreads();
  // back substitution, one warp per right-hand-side column
  for (int r = warp; r < nb; r += nwarps) {
    double *col = B + (size_t)r * ldb;
    for (int j = m - 1; j >= 0; --j) {
      const double xj = col[j] / A[j + (size_t)j * lda];
      __syncwarp();
      if (lane == 0) col[j] = xj;
      for (int i = lane; i < j; i += 32) col[i] -= A[i + (size_t)j * lda] * xj;
      __syncwarp();
    }
  }
  __syncthreads();
  return true;
}

// ----------------------------------------------------- warp LU solve (apply)
// x <- A^{-1} x for a factored m x m block (packed L\U + pivots) held in
// global memory; x lives in a per-warp shared buffer. Mirrors
// LUFactors::Solve (interchanges, unit-lower forward, upper backward).
__device__ __forceinline__ void warp_lu_apply(const double *__restrict__ lu, const int *__restrict__ piv,
                                              int m, double *x) {
  const int lane = threadIdx.x & 31;
  if (lane == 0)
    for (int i = 0; i < m; ++i) {
      const int p = piv[i];
      if (p != i) {
        const double t = x[i];
        x[i] = x[p];
        x[p] = t;
      }
    }
  __syncwarp();
  for (int j = 0; j < m; ++j) {
    const double xj = x[j];
    for (int i = j + 1 + lane; i < m; i += 32) x[i] -= lu[i + (size_t)j * m] * xj;
    __syncwarp();
  }
  for (int j = m - 1; j >= 0; --j) {
    const double xj = x[j] / lu[j + (size_t)j * m];
    __syncwarp();
    if (lane == 0) x[j] = xj;
    for (int i = lane; i < j; i += 32) x[i] -= lu[i + (size_t)j * m] * xj;
    __syncwarp();
  }
}

}  // namespace eg
