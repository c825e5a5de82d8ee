// Cell-local kernels of the DG discretisation: frozen HLL bounds, admissibility,
// the weak residual and its partially assembled Jacobian action (one fused
// sum-factorised kernel), and the DG block-Jacobi build/factor/apply.
//
// Data layout (device): body vectors u[e*m + 4*i + c] with cells row-major and
// nodes lexicographic; one thread owns one (cell, node) and its 4 components.
// Neighbour traces are read straight from global memory (L1/L2 resident: each
// cell's lines are re-read by at most its four neighbours), so no face buffer
// round trip through HBM is needed.
#include "eg_cellmat.cuh"
#include "eg_internal.h"

namespace eg {

template <int Q>
struct CellCfg {
  static constexpr int P = Q * Q;
  static constexpr int M = 4 * P;
  static constexpr int CPB = (256 / P) < 64 ? (256 / P) : 64;  // cells per block
  static constexpr int THREADS = CPB * P;
};

// ------------------------------------------------------------------ Freeze
// One thread per face point (src/problem.cpp:357-374 and WaveRate 377-384).
template <int Q>
__global__ void __launch_bounds__(256) freeze_kernel(Geo g, const double *__restrict__ tab,
                                                     const double *__restrict__ u, double *fa,
                                                     double *fb, double *flw, double *frw,
                                                     double *fpen, double *D, int *err,
                                                     unsigned long long *wave) {
  __shared__ STab<Q> st;
  __shared__ double red[256];
  load_tables<Q>(st, tab);
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  double speed = 0.;
  if (idx < g.nf * Q) {
    const int f = idx / Q, j = idx % Q, c = f >> 1, axis = f & 1;
    const int R = neighbour(c, axis == 0 ? 1 : 3, g.nx, g.ny);
    double ul[4], ur[4];
    trace4<Q>(st, u, c, axis == 0 ? 1 : 3, j, ul);
    trace4<Q>(st, u, R, axis == 0 ? 0 : 2, j, ur);
    double a = 0., b = 0.;
    const int code = hll_speeds(ul, ur, axis, g.gamma, g.gm1, g.safety, a, b);
    if (code != DERR_NONE) {
      raise_err(err, code);
    } else if (!(a + b > 0)) {
      raise_err(err, DERR_DEGENERATE_HLL);
    }
    const double inv = 1. / (a + b);
    fa[idx] = a;
    fb[idx] = b;
    flw[idx] = b * inv;
    frw[idx] = a * inv;
    fpen[idx] = a * b * inv;
    if (D) {
      const double diag = st.ew(j) * (a + b);
      double *dd = D + (size_t)f * (4 * Q) + 4 * j;
      dd[0] = dd[1] = dd[2] = dd[3] = diag;
    }
    speed = fmax(a, b);
  }
  red[threadIdx.x] = speed;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  // non-negative doubles order like their bit patterns
  if (threadIdx.x == 0) atomicMax(wave, (unsigned long long)__double_as_longlong(red[0]));
}

// ------------------------------------------------------------- Admissible
// Positivity at every volume node and face point (src/problem.cpp:259-275).
template <int Q>
__global__ void __launch_bounds__(256) admissible_kernel(Geo g, const double *__restrict__ tab,
                                                         const double *__restrict__ u, int *flag) {
  using C = CellCfg<Q>;
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const int lc = threadIdx.x / C::P, node = threadIdx.x % C::P;
  const int e = blockIdx.x * C::CPB + lc;
  if (lc >= C::CPB || e >= g.n) return;
  bool ok = true;
  {
    const double *v = u + (size_t)e * C::M + 4 * node;
    const double s[4] = {v[0], v[1], v[2], v[3]};
    ok = positive(s, g.gm1);
  }
  for (int task = node; task < 4 * Q; task += C::P) {
    double s[4];
    trace4<Q>(st, u, e, task / Q, task % Q, s);
    ok = ok && positive(s, g.gm1);
  }
  if (!ok) *flag = 0;
}

// -------------------------------------------- residual / Jacobian action
// Single-kernel forms, every cell evaluating its own face points (each face
// point twice). MODE 1 serves the single Jacobian actions; the residual runs
// as residual_face_kernel + residual_cell_kernel below, with the same
// arithmetic.
// MODE 0: r = M^{-1}[-dt sum_q w (Gx F_x + Gy F_y) + lifted HLL fluxes] + u - old
//         (Problem::Residual, src/problem.cpp:445-507);
// MODE 1: y = x + M^{-1}[-D_x^T(dt w J_x x) - D_y^T(dt w J_y x) + face lift of
//         (lw J(U_L) + pen) x_L + (rw J(U_R) - pen) x_R]
//         (PartialDGOperator::Mult, src/partial.cpp:62-135), with the flux
//         Jacobians recomputed from the Newton state instead of cached.
template <int Q, int MODE>
__global__ void __launch_bounds__(CellCfg<Q>::THREADS)
    cell_operator_kernel(Geo g, const double *__restrict__ tab, Frozen fz,
                         const double *__restrict__ u, const double *__restrict__ x_or_old,
                         double *__restrict__ out) {
  using C = CellCfg<Q>;
  constexpr int P = C::P, M = C::M, CPB = C::CPB;
  __shared__ STab<Q> st;
  __shared__ double fxs[CPB][P][4], fys[CPB][P][4];
  __shared__ double hs[CPB][4 * Q][4];
  load_tables<Q>(st, tab);
  __syncthreads();
  const int lc = threadIdx.x / P, node = threadIdx.x % P;
  const int e = blockIdx.x * CPB + lc;
  const bool active = lc < CPB && e < g.n;
  double uu[4] = {0., 0., 0., 0.}, xx[4] = {0., 0., 0., 0.};
  if (active) {
    const double *v = u + (size_t)e * M + 4 * node;
#pragma unroll
    for (int c = 0; c < 4; ++c) uu[c] = v[c];
    const double *xv = x_or_old + (size_t)e * M + 4 * node;
#pragma unroll
    for (int c = 0; c < 4; ++c) xx[c] = xv[c];
    const double wdt = g.dt * st.w(node);
    double fx[4], fy[4];
    if (MODE == 0) {
      flux(uu, 0, g.gm1, fx);
      flux(uu, 1, g.gm1, fy);
    } else {
      double j[16];
      jacobian(uu, 0, g.gm1, j);
      mat4_vec(j, xx, fx);
      jacobian(uu, 1, g.gm1, j);
      mat4_vec(j, xx, fy);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      fxs[lc][node][c] = wdt * fx[c];
      fys[lc][node][c] = wdt * fy[c];
    }
  }
  if (lc < CPB && e < g.n) {
    for (int task = node; task < 4 * Q; task += P) {
      const int s = task / Q, j = task % Q;
      const bool own_left = side_is_left(s);
      const int nb = neighbour(e, s, g.nx, g.ny);
      const int cl = own_left ? e : nb, cr = own_left ? nb : e;
      const int sl = s < 2 ? 1 : 3, sr = sl - 1;
      const int axis = s < 2 ? 0 : 1;
      const int f = own_left ? 2 * e + axis : 2 * nb + axis;
      const int fi = f * Q + j;
      double ul[4], ur[4], h[4];
      trace4<Q>(st, u, cl, sl, j, ul);
      trace4<Q>(st, u, cr, sr, j, ur);
      const double lw = fz.lw[fi], rw = fz.rw[fi], pen = fz.pen[fi];
      if (MODE == 0) {
        double fl[4], fr[4];
        flux(ul, axis, g.gm1, fl);
        flux(ur, axis, g.gm1, fr);
#pragma unroll
        for (int c = 0; c < 4; ++c) h[c] = lw * fl[c] + rw * fr[c] + pen * (ul[c] - ur[c]);
      } else {
        double xl[4], xr[4], jl[16], jr[16], zl[4], zr[4];
        trace4<Q>(st, x_or_old, cl, sl, j, xl);
        trace4<Q>(st, x_or_old, cr, sr, j, xr);
        jacobian(ul, axis, g.gm1, jl);
        jacobian(ur, axis, g.gm1, jr);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          jl[k] *= lw;
          jr[k] *= rw;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          jl[c * 5] += pen;
          jr[c * 5] -= pen;
        }
        mat4_vec(jl, xl, zl);
        mat4_vec(jr, xr, zr);
#pragma unroll
        for (int c = 0; c < 4; ++c) h[c] = zl[c] + zr[c];
      }
      const double len = axis == 0 ? g.hy : g.hx;
      const double scale = g.dt * len / g.area * st.ew(j);
      const double sg = own_left ? scale : -scale;
#pragma unroll
      for (int c = 0; c < 4; ++c) hs[lc][task][c] = sg * h[c];
    }
  }
  __syncthreads();
  if (!active) return;
  const int ix = node % Q, iy = node / Q;
  double acc[4] = {0., 0., 0., 0.};
#pragma unroll
  for (int a = 0; a < Q; ++a) {
    const double dx = st.tdx(a, ix), dy = st.tdy(a, iy);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += dx * fxs[lc][iy * Q + a][c] + dy * fys[lc][a * Q + ix][c];
  }
  const double w0 = st.fb(0, iy, ix), w1 = st.fb(1, iy, ix);
  const double w2 = st.fb(2, ix, iy), w3 = st.fb(3, ix, iy);
  const double im = st.inv_mass(node);
  double *o = out + (size_t)e * M + 4 * node;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double face = w0 * hs[lc][0 * Q + iy][c] + w1 * hs[lc][1 * Q + iy][c] +
                        w2 * hs[lc][2 * Q + ix][c] + w3 * hs[lc][3 * Q + ix][c];
    const double v = im * (face - acc[c]);
    o[c] = MODE == 0 ? v + uu[c] - xx[c] : v + xx[c];
  }
}

// ------------------------------------ DG partial assembly: Refresh + Mult
// PartialDGOperator::Refresh (src/partial.cpp:31-59) caches, once per
// Newton state, the scaled flux Jacobians the action needs: per cell node
// dt w J_x(u) and dt w J_y(u), per face point lw J(U_L) + pen I and
// rw J(U_R) - pen I. Both caches are stored component-major (entry k of
// every node, then entry k + 1, ...; k = row + 4 col of a column-major 4x4
// block, J_x before J_y, the left block before the right), so that
// consecutive threads read
// consecutive doubles. The cached action (PartialDGOperator::Mult,
// src/partial.cpp:62-135) then streams x, y and the caches once, which is
// the byte count the partial-assembly roofline is scored against, instead
// of recomputing the Jacobians (a flux Jacobian and two face traces per
// point) in every Krylov iteration.
template <int Q>
__global__ void __launch_bounds__(256) dg_refresh_volume_kernel(Geo g, const double *__restrict__ tab,
                                                                const double *__restrict__ u,
                                                                double *__restrict__ vol) {
  constexpr int P = Q * Q, M = 4 * P;
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const long long np = (long long)g.n * P;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < np;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long e = idx / P;
    const int node = (int)(idx % P);
    double uu[4], j[16];
#pragma unroll
    for (int c = 0; c < 4; ++c) uu[c] = u[e * M + 4 * node + c];
    const double wdt = g.dt * st.w(node);
    jacobian(uu, 0, g.gm1, j);
#pragma unroll
    for (int k = 0; k < 16; ++k) vol[k * np + idx] = wdt * j[k];
    jacobian(uu, 1, g.gm1, j);
#pragma unroll
    for (int k = 0; k < 16; ++k) vol[(16 + k) * np + idx] = wdt * j[k];
  }
}

template <int Q>
__global__ void __launch_bounds__(256) dg_refresh_face_kernel(Geo g, const double *__restrict__ tab, Frozen fz,
                                                              const double *__restrict__ u,
                                                              double *__restrict__ face) {
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const long long nq = (long long)g.nf * Q;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nq;
       idx += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(idx / Q), j = (int)(idx % Q);
    const int L = f >> 1, axis = f & 1;
    const int sl = axis ? 3 : 1, sr = sl - 1;
    const int R = neighbour(L, sl, g.nx, g.ny);
    double ul[4], ur[4], jl[16], jr[16];
    trace4<Q>(st, u, L, sl, j, ul);
    trace4<Q>(st, u, R, sr, j, ur);
    jacobian(ul, axis, g.gm1, jl);
    jacobian(ur, axis, g.gm1, jr);
    const double lw = fz.lw[idx], rw = fz.rw[idx], pen = fz.pen[idx];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const bool diag = (k % 5) == 0;
      face[k * nq + idx] = lw * jl[k] + (diag ? pen : 0.);
      face[(16 + k) * nq + idx] = rw * jr[k] - (diag ? pen : 0.);
    }
  }
}

// Face part of the cached action, once per face point: h = scale (jl x_L +
// jr x_R) with x_L, x_R the traces of x on the face's two cells and
// scale = dt |face| / |K| ew_j (added with + into the left cell, - into the
// right one by dg_cached_apply_kernel).
template <int Q>
__global__ void __launch_bounds__(256) dg_cached_face_kernel(Geo g, const double *__restrict__ tab,
                                                             const double *__restrict__ face,
                                                             const double *__restrict__ x,
                                                             double *__restrict__ hface) {
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const long long nq = (long long)g.nf * Q;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nq;
       idx += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(idx / Q), j = (int)(idx % Q);
    const int L = f >> 1, axis = f & 1;
    const int sl = axis ? 3 : 1, sr = sl - 1;
    const int R = neighbour(L, sl, g.nx, g.ny);
    double xl[4], xr[4], h[4] = {0., 0., 0., 0.};
    trace4<Q>(st, x, L, sl, j, xl);
    trace4<Q>(st, x, R, sr, j, xr);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c)
        h[r] += __ldcs(face + (r + 4 * c) * nq + idx) * xl[c] + __ldcs(face + (16 + r + 4 * c) * nq + idx) * xr[c];
    const double len = axis == 0 ? g.hy : g.hx;
    const double scale = g.dt * len / g.area * st.ew(j);
    double4 o;
    o.x = scale * h[0];
    o.y = scale * h[1];
    o.z = scale * h[2];
    o.w = scale * h[3];
    reinterpret_cast<double4 *>(hface)[idx] = o;
  }
}

// y = x + M^{-1}[-D_x^T(jx x) - D_y^T(jy x) + face lift of (jl x_L + jr x_R)]
// with the cached jx, jy and the face values of dg_cached_face_kernel (one
// thread per node, CellCfg<Q>::CPB cells per CTA).
template <int Q>
__global__ void __launch_bounds__(CellCfg<Q>::THREADS)
    dg_cached_apply_kernel(Geo g, const double *__restrict__ tab, const double *__restrict__ vol,
                           const double *__restrict__ hface, const double *__restrict__ x, double *__restrict__ out) {
  using C = CellCfg<Q>;
  constexpr int P = C::P, M = C::M, CPB = C::CPB;
  __shared__ STab<Q> st;
  __shared__ double fxs[CPB][P][4], fys[CPB][P][4];
  __shared__ double hs[CPB][4 * Q][4];
  load_tables<Q>(st, tab);
  __syncthreads();
  const int lc = threadIdx.x / P, node = threadIdx.x % P;
  const int e = blockIdx.x * CPB + lc;
  const bool active = lc < CPB && e < g.n;
  const long long np = (long long)g.n * P;
  double xx[4] = {0., 0., 0., 0.};
  if (active) {
    const double *xv = x + (size_t)e * M + 4 * node;
#pragma unroll
    for (int c = 0; c < 4; ++c) xx[c] = xv[c];
    const long long idx = (long long)e * P + node;
    double fx[4] = {0., 0., 0., 0.}, fy[4] = {0., 0., 0., 0.};
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        fx[r] += __ldcs(vol + (r + 4 * c) * np + idx) * xx[c];  // column-major 4x4
        fy[r] += __ldcs(vol + (16 + r + 4 * c) * np + idx) * xx[c];
      }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      fxs[lc][node][c] = fx[c];
      fys[lc][node][c] = fy[c];
    }
  }
  if (active) {
    for (int task = node; task < 4 * Q; task += P) {
      const int s = task / Q, j = task % Q;
      const bool own_left = side_is_left(s);
      const int nb = neighbour(e, s, g.nx, g.ny);
      const int axis = s < 2 ? 0 : 1;
      const int f = own_left ? 2 * e + axis : 2 * nb + axis;
      const double4 h = reinterpret_cast<const double4 *>(hface)[(size_t)f * Q + j];
      const double sg = own_left ? 1. : -1.;
      hs[lc][task][0] = sg * h.x;
      hs[lc][task][1] = sg * h.y;
      hs[lc][task][2] = sg * h.z;
      hs[lc][task][3] = sg * h.w;
    }
  }
  __syncthreads();
  if (!active) return;
  const int ix = node % Q, iy = node / Q;
  double acc[4] = {0., 0., 0., 0.};
#pragma unroll
  for (int a = 0; a < Q; ++a) {
    const double dx = st.tdx(a, ix), dy = st.tdy(a, iy);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += dx * fxs[lc][iy * Q + a][c] + dy * fys[lc][a * Q + ix][c];
  }
  const double w0 = st.fb(0, iy, ix), w1 = st.fb(1, iy, ix);
  const double w2 = st.fb(2, ix, iy), w3 = st.fb(3, ix, iy);
  const double im = st.inv_mass(node);
  double *o = out + (size_t)e * M + 4 * node;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double fc = w0 * hs[lc][0 * Q + iy][c] + w1 * hs[lc][1 * Q + iy][c] + w2 * hs[lc][2 * Q + ix][c] +
                      w3 * hs[lc][3 * Q + ix][c];
    o[c] = im * (fc - acc[c]) + xx[c];
  }
}

// Residual face part, once per face point: h = scale (lw F(U_L) + rw F(U_R)
// + pen (U_L - U_R)) with U_L, U_R the traces on the face's two cells and
// scale = dt |face| / |K| ew_j (Problem::Residual's numerical flux,
// src/problem.cpp:470-495; added with + into the left cell, - into the right
// one). The same arithmetic as the cell-side evaluation it replaces, which
// computed every face point twice.
template <int Q>
__global__ void __launch_bounds__(256) residual_face_kernel(Geo g, const double *__restrict__ tab, Frozen fz,
                                                            const double *__restrict__ u, double *__restrict__ hface) {
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const long long nq = (long long)g.nf * Q;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nq;
       idx += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(idx / Q), j = (int)(idx % Q);
    const int L = f >> 1, axis = f & 1;
    const int sl = axis ? 3 : 1, sr = sl - 1;
    const int R = neighbour(L, sl, g.nx, g.ny);
    double ul[4], ur[4], fl[4], fr[4];
    trace4<Q>(st, u, L, sl, j, ul);
    trace4<Q>(st, u, R, sr, j, ur);
    flux(ul, axis, g.gm1, fl);
    flux(ur, axis, g.gm1, fr);
    const double lw = fz.lw[idx], rw = fz.rw[idx], pen = fz.pen[idx];
    const double len = axis == 0 ? g.hy : g.hx;
    const double scale = g.dt * len / g.area * st.ew(j);
    double h[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) h[c] = scale * (lw * fl[c] + rw * fr[c] + pen * (ul[c] - ur[c]));
    reinterpret_cast<double4 *>(hface)[idx] = make_double4(h[0], h[1], h[2], h[3]);
  }
}

// r = M^{-1}[-dt sum_q w (Gx F_x + Gy F_y) + lifted face values] + u - old
// with the face values of residual_face_kernel (one thread per node,
// CellCfg<Q>::CPB cells per CTA).
template <int Q>
__global__ void __launch_bounds__(CellCfg<Q>::THREADS)
    residual_cell_kernel(Geo g, const double *__restrict__ tab, const double *__restrict__ u,
                         const double *__restrict__ old, const double *__restrict__ hface, double *__restrict__ out) {
  using C = CellCfg<Q>;
  constexpr int P = C::P, M = C::M, CPB = C::CPB;
  __shared__ STab<Q> st;
  __shared__ double fxs[CPB][P][4], fys[CPB][P][4];
  __shared__ double hs[CPB][4 * Q][4];
  load_tables<Q>(st, tab);
  __syncthreads();
  const int lc = threadIdx.x / P, node = threadIdx.x % P;
  const int e = blockIdx.x * CPB + lc;
  const bool active = lc < CPB && e < g.n;
  double uu[4] = {0., 0., 0., 0.}, oo[4] = {0., 0., 0., 0.};
  if (active) {
    const double *v = u + (size_t)e * M + 4 * node;
    const double *ov = old + (size_t)e * M + 4 * node;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uu[c] = v[c];
      oo[c] = ov[c];
    }
    const double wdt = g.dt * st.w(node);
    double fx[4], fy[4];
    flux(uu, 0, g.gm1, fx);
    flux(uu, 1, g.gm1, fy);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      fxs[lc][node][c] = wdt * fx[c];
      fys[lc][node][c] = wdt * fy[c];
    }
    for (int task = node; task < 4 * Q; task += P) {
      const int s = task / Q, j = task % Q;
      const bool own_left = side_is_left(s);
      const int nb = neighbour(e, s, g.nx, g.ny);
      const int axis = s < 2 ? 0 : 1;
      const int f = own_left ? 2 * e + axis : 2 * nb + axis;
      const double4 h = reinterpret_cast<const double4 *>(hface)[(size_t)f * Q + j];
      const double sg = own_left ? 1. : -1.;
      hs[lc][task][0] = sg * h.x;
      hs[lc][task][1] = sg * h.y;
      hs[lc][task][2] = sg * h.z;
      hs[lc][task][3] = sg * h.w;
    }
  }
  __syncthreads();
  if (!active) return;
  const int ix = node % Q, iy = node / Q;
  double acc[4] = {0., 0., 0., 0.};
#pragma unroll
  for (int a = 0; a < Q; ++a) {
    const double dx = st.tdx(a, ix), dy = st.tdy(a, iy);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] += dx * fxs[lc][iy * Q + a][c] + dy * fys[lc][a * Q + ix][c];
  }
  const double w0 = st.fb(0, iy, ix), w1 = st.fb(1, iy, ix);
  const double w2 = st.fb(2, ix, iy), w3 = st.fb(3, ix, iy);
  const double im = st.inv_mass(node);
  double *o = out + (size_t)e * M + 4 * node;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double fc = w0 * hs[lc][0 * Q + iy][c] + w1 * hs[lc][1 * Q + iy][c] + w2 * hs[lc][2 * Q + ix][c] +
                      w3 * hs[lc][3 * Q + ix][c];
    const double v = im * (fc - acc[c]);
    o[c] = v + uu[c] - oo[c];
  }
}

template <int Q>
__host__ __device__ constexpr int lu_rmax() {
  return (4 * Q * Q + 31) / 32;
}
// Cells whose m x m block (plus staging) fits in shared memory.
template <int Q>
__host__ __device__ constexpr bool dg_block_in_smem() {
  return 4 * Q * Q <= 144;
}

// ------------------------------------------------------ DG block Jacobi
// Per cell: diagonal block (volume + own-face HLL terms) built at the Newton
// state, then factored in place with partial pivoting (linear.cpp:198-202).
template <int Q>
__global__ void __launch_bounds__(256)
    dg_jacobi_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                     double *blocks, int *pivots, bool factor, int *err) {
  constexpr int P = Q * Q, M = 4 * P;
  constexpr bool SM = dg_block_in_smem<Q>();
  __shared__ STab<Q> st;
  __shared__ double us[M], UT[16 * Q], FM[4 * Q * 16];
  __shared__ int piv_s[M];
  __shared__ double inv_piv[M];
  __shared__ double bcast[2];
  extern __shared__ double dyn[];
  load_tables<Q>(st, tab);
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    for (int i = threadIdx.x; i < M; i += blockDim.x) us[i] = u[(size_t)e * M + i];
    __syncthreads();
    cell_traces<Q>(st, us, UT);
    __syncthreads();
    dg_face_matrices<Q>(UT, FM, g, fz, e);
    __syncthreads();
    double *A = SM ? dyn : blocks + (size_t)e * M * M;
    build_cell_matrix<Q>(A, M, st, us, FM, g);
    __syncthreads();
    if (factor) {
      const bool ok = cta_lu_solve<lu_rmax<Q>()>(A, M, nullptr, 1, M, 0, piv_s, inv_piv, bcast);
      if (!ok && threadIdx.x == 0) raise_err(err, DERR_SINGULAR_JACOBI);
    } else {
      for (int i = threadIdx.x; i < M; i += blockDim.x) piv_s[i] = i;
    }
    __syncthreads();
    if (SM) {
      double *dst = blocks + (size_t)e * M * M;
      for (int i = threadIdx.x; i < M * M; i += blockDim.x) dst[i] = A[i];
    }
    for (int i = threadIdx.x; i < M; i += blockDim.x) pivots[(size_t)e * M + i] = piv_s[i];
  }
}

// --------------------------------------------------------- block LU apply
// x_b = LU_b^{-1} b_b for every block (one warp per block); Jacobi apply of
// LinearSolver::Impl::Precondition (src/linear.cpp:66-75).
__global__ void __launch_bounds__(256) block_apply_kernel(const double *__restrict__ blocks,
                                                          const int *__restrict__ piv, int nblocks,
                                                          int bs, const double *__restrict__ b,
                                                          double *__restrict__ x) {
  extern __shared__ double xs[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * (blockDim.x >> 5) + warp;
  if (blk >= nblocks) return;
  double *v = xs + warp * bs;
  for (int i = lane; i < bs; i += 32) v[i] = b[(size_t)blk * bs + i];
  __syncwarp();
  warp_lu_apply(blocks + (size_t)blk * bs * bs, piv + (size_t)blk * bs, bs, v);
  for (int i = lane; i < bs; i += 32) x[(size_t)blk * bs + i] = v[i];
}

// The same apply with the block's part of x in registers (lane holds rows
// lane + 32 r, r < R): sweep steps communicate through shuffles only. Every
// step reads one column of the factor; those reads do not depend on x, so
// they are issued PD steps ahead into a register ring (fully unrolled sweeps,
// static ring slots) and a step no longer waits out a memory latency. Column
// and row indices are clamped into the block for the loads; only the
// updates are predicated. The diagonal is applied as a product with its
// reciprocal.
template <int R>
__global__ void __launch_bounds__(256) block_apply_reg_kernel(const double *__restrict__ blocks,
                                                              const int *__restrict__ piv, int nblocks,
                                                              int m, const double *__restrict__ b,
                                                              double *__restrict__ x) {
  constexpr int S = 32 * R;                             // sweep steps (j >= m are no-ops)
  constexpr int PD = R == 1 ? 16 : (R == 2 ? 8 : (R <= 4 ? 4 : (R <= 8 ? 2 : 1)));  // columns per chunk
  extern __shared__ double xs[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * (blockDim.x >> 5) + warp;
  if (blk >= nblocks) return;
  double *v = xs + (size_t)warp * m;
  const double *lu = blocks + (size_t)blk * m * m;
  const int *pv = piv + (size_t)blk * m;
  for (int i = lane; i < m; i += 32) v[i] = b[(size_t)blk * m + i];
  __syncwarp();
  if (lane == 0)
    for (int i = 0; i < m; ++i) {  // row exchanges of the factorisation, in order
      const int p = pv[i];
      if (p != i) {
        const double t = v[i];
        v[i] = v[p];
        v[p] = t;
      }
    }
  __syncwarp();
  double xr[R];
#pragma unroll
  for (int r = 0; r < R; ++r) xr[r] = lane + 32 * r < m ? v[lane + 32 * r] : 0.;
  int rows[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rows[r] = min(lane + 32 * r, m - 1);
  auto load_col = [&](double (&dst)[R], int j) {
    const double *col = lu + (size_t)min(max(j, 0), m - 1) * m;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r] = col[rows[r]];
  };
  // columns are read in chunks of PD: the next chunk's loads are issued
  // before the current chunk's steps (double buffer in registers)
  double cur[PD][R], nxt[PD][R];
  // forward: unit lower triangle, columns 0, 1, ...
#pragma unroll
  for (int d = 0; d < PD; ++d) load_col(cur[d], d);
#pragma unroll
  for (int jb = 0; jb < R; ++jb) {
#pragma unroll 1
    for (int cc = 0; cc < 32 / PD; ++cc) {
      const int j0 = 32 * jb + PD * cc;
#pragma unroll
      for (int d = 0; d < PD; ++d) load_col(nxt[d], j0 + PD + d);
#pragma unroll
      for (int d = 0; d < PD; ++d) {
        const int j = j0 + d;
        const double xj = __shfl_sync(0xffffffffu, xr[jb], PD * cc + d);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + 32 * r;
          xr[r] = (j < m && i > j && i < m) ? xr[r] - cur[d][r] * xj : xr[r];
        }
      }
#pragma unroll
      for (int d = 0; d < PD; ++d)
#pragma unroll
        for (int r = 0; r < R; ++r) cur[d][r] = nxt[d][r];
    }
  }
  // backward: upper triangle with its diagonal, columns S-1, S-2, ...
#pragma unroll
  for (int d = 0; d < PD; ++d) load_col(cur[d], S - 1 - d);
#pragma unroll
  for (int jb = R - 1; jb >= 0; --jb) {
#pragma unroll 1
    for (int cc = 32 / PD - 1; cc >= 0; --cc) {
      const int jtop = 32 * jb + PD * cc + PD - 1;  // first (highest) column of the chunk
#pragma unroll
      for (int d = 0; d < PD; ++d) load_col(nxt[d], jtop - PD - d);
#pragma unroll
      for (int d = 0; d < PD; ++d) {
        const int j = jtop - d;
        const int jl = PD * cc + PD - 1 - d;  // j % 32
        // u_jj sits in lane j % 32, register j / 32 (= jb) of this column
        const double ujj = __shfl_sync(0xffffffffu, cur[d][jb], jl);
        const double xo = __shfl_sync(0xffffffffu, xr[jb], jl) * (1.0 / ujj);
        if (j < m && lane == jl) xr[jb] = xo;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = lane + 32 * r;
          xr[r] = (j < m && i < j) ? xr[r] - cur[d][r] * xo : xr[r];
        }
      }
#pragma unroll
      for (int d = 0; d < PD; ++d)
#pragma unroll
        for (int r = 0; r < R; ++r) cur[d][r] = nxt[d][r];
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (lane + 32 * r < m) x[(size_t)blk * m + lane + 32 * r] = xr[r];
}

// ================================================================ launchers
static Frozen frozen_of(Ctx &c) { return Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}; }

void launch_freeze(Ctx &c, const double *u, bool check_admissible) {
  if (check_admissible) {
    launch_admissible(c, u);
    EG_CUDA(cudaMemcpyAsync(c.herr + 1, c.derr + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (!c.herr[1]) fail(EG_ERR_INADMISSIBLE, "Old state is inadmissible; refine mesh");
  }
  EG_CUDA(cudaMemsetAsync(c.dscal + DS_WAVE, 0, sizeof(double), c.stream));
  const int total = c.nf * c.q;
  const int blocks = (total + 255) / 256;
  ProfScope ps(c, EG_K_FREEZE, 1);
  EG_DISPATCH_Q(c.q, freeze_kernel<Q><<<blocks, 256, 0, c.stream>>>(
                         c.geo, c.tab, u, c.fa, c.fbb, c.flw, c.frw, c.fpen, c.D, c.derr,
                         reinterpret_cast<unsigned long long *>(c.dscal + DS_WAVE)));
  EG_CUDA(cudaGetLastError());
}

void launch_admissible(Ctx &c, const double *u) {
  const int one = 1;
  EG_CUDA(cudaMemcpyAsync(c.derr + 1, &one, sizeof(int), cudaMemcpyHostToDevice, c.stream));
  ProfScope ps(c, EG_K_ADMISSIBLE, 1);
  EG_DISPATCH_Q(c.q, {
    using C = CellCfg<Q>;
    const int blocks = (c.n + C::CPB - 1) / C::CPB;
    admissible_kernel<Q><<<blocks, C::THREADS, 0, c.stream>>>(c.geo, c.tab, u, c.derr + 1);
  });
  EG_CUDA(cudaGetLastError());
}

static int sm_count();

void launch_residual(Ctx &c, const double *u, const double *old, double *r) {
  ProfScope ps(c, EG_K_RESIDUAL, 2);
  if (!c.dgc_h) c.dgc_h = c.alloc_n<double>((size_t)4 * c.nf * c.q);
  const int grid = (int)std::min<long long>(((long long)c.nf * c.q + 255) / 256, (long long)sm_count() * 16);
  EG_DISPATCH_Q(c.q, {
    using C = CellCfg<Q>;
    const int blocks = (c.n + C::CPB - 1) / C::CPB;
    residual_face_kernel<Q><<<grid, 256, 0, c.stream>>>(c.geo, c.tab, frozen_of(c), u, c.dgc_h);
    residual_cell_kernel<Q><<<blocks, C::THREADS, 0, c.stream>>>(c.geo, c.tab, u, old, c.dgc_h, r);
  });
  EG_CUDA(cudaGetLastError());
}

void launch_dg_refresh(Ctx &c, const double *u) {
  ProfScope ps(c, EG_K_DG_APPLY, 1);
  if (!c.dgc_vol) {
    c.dgc_vol = c.alloc_n<double>((size_t)32 * c.n * c.p);
    c.dgc_face = c.alloc_n<double>((size_t)32 * c.nf * c.q);
  }
  const int grid = sm_count() * 8;
  EG_DISPATCH_Q(c.q, {
    dg_refresh_volume_kernel<Q><<<grid, 256, 0, c.stream>>>(c.geo, c.tab, u, c.dgc_vol);
    dg_refresh_face_kernel<Q><<<grid, 256, 0, c.stream>>>(c.geo, c.tab, frozen_of(c), u, c.dgc_face);
  });
  EG_CUDA(cudaGetLastError());
}

void launch_dg_apply_cached(Ctx &c, const double *x, double *y) {
  if (!c.dgc_vol) fail(EG_ERR_INVALID, "DG partial assembly used before its refresh");
  ProfScope ps(c, EG_K_DG_APPLY, 1);
  if (!c.dgc_h) c.dgc_h = c.alloc_n<double>((size_t)4 * c.nf * c.q);
  const int grid = (int)std::min<long long>(((long long)c.nf * c.q + 255) / 256, (long long)sm_count() * 16);
  EG_DISPATCH_Q(c.q, {
    using C = CellCfg<Q>;
    const int blocks = (c.n + C::CPB - 1) / C::CPB;
    dg_cached_face_kernel<Q><<<grid, 256, 0, c.stream>>>(c.geo, c.tab, c.dgc_face, x, c.dgc_h);
    dg_cached_apply_kernel<Q><<<blocks, C::THREADS, 0, c.stream>>>(c.geo, c.tab, c.dgc_vol, c.dgc_h, x, y);
  });
  EG_CUDA(cudaGetLastError());
}

void launch_dg_apply(Ctx &c, const double *u, const double *x, double *y) {
  ProfScope ps(c, EG_K_DG_APPLY, 1);
  EG_DISPATCH_Q(c.q, {
    using C = CellCfg<Q>;
    const int blocks = (c.n + C::CPB - 1) / C::CPB;
    cell_operator_kernel<Q, 1><<<blocks, C::THREADS, 0, c.stream>>>(c.geo, c.tab, frozen_of(c), u,
                                                                     x, y);
  });
  EG_CUDA(cudaGetLastError());
}

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

void launch_dg_jacobi(Ctx &c, const double *u, bool factor) {
  if (factor && dg_inverse_supported(c.q)) {
    launch_dg_inverse(c, u);
    c.dg_pc_inverse = true;
    return;
  }
  c.dg_pc_inverse = false;
  c.ensure_pc_dg();
  ProfScope ps(c, EG_K_DG_JACOBI, 1);
  EG_DISPATCH_Q(c.q, {
    constexpr int M = 4 * Q * Q;
    const size_t dyn = dg_block_in_smem<Q>() ? sizeof(double) * M * M : 0;
    auto kern = dg_jacobi_kernel<Q>;
    if (dyn > 48 * 1024)
      EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    const int grid = std::min(c.n, sm_count() * 8);
    kern<<<grid, 256, dyn, c.stream>>>(c.geo, c.tab, frozen_of(c), u, c.pc_dg, c.piv_dg, factor, c.derr);
  });
  EG_CUDA(cudaGetLastError());
}

void launch_dg_jacobi_apply(Ctx &c, const double *b, double *x) {
  if (c.dg_pc_inverse)
    launch_dg_inverse_apply(c, b, x);
  else
    launch_block_apply(c, c.pc_dg, c.piv_dg, c.n, c.m, b, x);
}

void launch_block_apply(Ctx &c, const double *blocks, const int *piv, int nblocks, int bs,
                        const double *b, double *x) {
  // 4 warps (blocks) per CTA: the register-resident sweeps use ~100
  // registers, so smaller CTAs pack more warps per SM
  const int warps = 4;
  const int grid = (nblocks + warps - 1) / warps;
  const size_t dyn = sizeof(double) * bs * warps;
  ProfScope ps(c, EG_K_PC_APPLY, 1);
  switch ((bs + 31) / 32) {
#define EG_BAR(RR)                                                                                    \
  case RR:                                                                                            \
    block_apply_reg_kernel<RR><<<grid, warps * 32, dyn, c.stream>>>(blocks, piv, nblocks, bs, b, x);   \
    break;
    EG_BAR(1) EG_BAR(2) EG_BAR(4) EG_BAR(5) EG_BAR(7) EG_BAR(8) EG_BAR(11)
#undef EG_BAR
    default:
      block_apply_kernel<<<grid, warps * 32, dyn, c.stream>>>(blocks, piv, nblocks, bs, b, x);
  }
  EG_CUDA(cudaGetLastError());
}

}  // namespace eg
