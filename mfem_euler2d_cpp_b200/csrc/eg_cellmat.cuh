// Cell-block assembly shared by DG block Jacobi and HDG condensation.
#pragma once
#include "eg_device.cuh"

namespace eg {
// ------------------------------------------------- cell Jacobian assembly
// Shared by DG block Jacobi and HDG condensation: the cell block
//   A = I + M^{-1}[volume Jacobian] + sum_faces scale*phi_i*M^{-1}_ii*phi_j*FM(s,j)
// (Problem::VolumeJacobianCell src/problem.cpp:519-550 plus the own-face terms
// of PartialDGOperator::DiagonalBlocks src/partial.cpp:265-298 or
// Problem::HybridCell src/problem.cpp:661-694). FM holds the signed 4x4 face
// matrices per (side, face point). One thread per column (trial node, comp).
template <int Q>
__device__ void build_cell_matrix(double *A, int lda, const STab<Q> &st, const double *us,
                                  const double *FM, const Geo &g) {
  constexpr int P = Q * Q, M = 4 * P;
  for (int col = threadIdx.x; col < M; col += blockDim.x) {
    double *a = A + (size_t)col * lda;
    for (int i = 0; i < M; ++i) a[i] = 0.;
    const int jn = col >> 2, d = col & 3;
    const int jx = jn % Q, jy = jn / Q;
    double jxm[16], jym[16];
    const double s4[4] = {us[4 * jn], us[4 * jn + 1], us[4 * jn + 2], us[4 * jn + 3]};
    jacobian(s4, 0, g.gm1, jxm);
    jacobian(s4, 1, g.gm1, jym);
    const double wdt = g.dt * st.w(jn);
    // x-line through jn (rows i = (ix, jy)); includes i == jn
    for (int ix = 0; ix < Q; ++ix) {
      const int i = jy * Q + ix;
      const double gx = st.tdx(jx, ix), gy = (ix == jx) ? st.tdy(jy, jy) : 0.;
      const double im = st.inv_mass(i);
#pragma unroll
      for (int c = 0; c < 4; ++c) a[4 * i + c] = -(wdt * (gx * jxm[c + 4 * d] + gy * jym[c + 4 * d])) * im;
    }
    // y-line through jn (rows i = (jx, iy)), i != jn
    for (int iy = 0; iy < Q; ++iy) {
      if (iy == jy) continue;
      const int i = iy * Q + jx;
      const double gy = st.tdy(jy, iy);
      const double im = st.inv_mass(i);
#pragma unroll
      for (int c = 0; c < 4; ++c) a[4 * i + c] = -(wdt * (gy * jym[c + 4 * d])) * im;
    }
    a[col] += 1.;
    // face terms
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int j = s < 2 ? jy : jx;      // face point of the line through jn
      const int lj = s < 2 ? jx : jy;     // position of jn along that line
      const double len = s < 2 ? g.hy : g.hx;
      const double scale = g.dt * len / g.area * st.ew(j);
      const double fbj = st.fb(s, j, lj);
      const double *fm = FM + (s * Q + j) * 16;
      for (int l = 0; l < Q; ++l) {
        const int i = line_node<Q>(s, j, l);
        const double wgt = scale * st.fb(s, j, l) * st.inv_mass(i) * fbj;
#pragma unroll
        for (int c = 0; c < 4; ++c) a[4 * i + c] += wgt * fm[c + 4 * d];
      }
    }
  }
}

// Signed DG face matrices of cell e from its traces UT: own-left sides add
// lw J(U_L) + pen I, own-right sides subtract rw J(U_R) - pen I
// (src/partial.cpp:272-294); FM[(s*Q+j)*16 + c + 4d].
template <int Q>
__device__ void dg_face_matrices(const double *UT, double *FM, const Geo &g, const Frozen &fz, int e) {
  for (int task = threadIdx.x; task < 4 * Q; task += blockDim.x) {
    const int s = task / Q, j = task % Q;
    const bool L = side_is_left(s);
    const int f = cell_face(e, s, g.nx, g.ny);
    const int fi = f * Q + j;
    double jm[16];
    jacobian(UT + 4 * task, s < 2 ? 0 : 1, g.gm1, jm);
    const double wgt = L ? fz.lw[fi] : fz.rw[fi], pen = fz.pen[fi];
    double *fm = FM + task * 16;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const bool diag = (k % 5) == 0;
      const double v = wgt * jm[k] + (diag ? (L ? pen : -pen) : 0.);
      fm[k] = L ? v : -v;
    }
  }
}

// Own traces of the cell at all 4Q face points into UT[(s*Q+j)*4 + c].
template <int Q>
__device__ void cell_traces(const STab<Q> &st, const double *us, double *UT) {
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
}

}  // namespace eg
