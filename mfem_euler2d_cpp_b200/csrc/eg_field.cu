// Device-side initial projection and diagnostics of the simple-wave problem:
// Problem::Initial (src/problem.cpp:329-349), Errors (704-726), Integral
// (727-738) and Differences (739-761), with the exact wave of
// EulerGas::exact (src/physics.cpp:64-93). A served request or a benchmark
// run then never moves its state across the host boundary between admission
// and result.
//
// One CTA per cell: the threads evaluate the exact wave at the points of the
// square Gauss-Legendre rule of order max(24, 2k+8) (13 x 13 points for
// k <= 8), then form the projection (each output node sums the points in the
// reference's order) or the cell's partial sums of the diagnostic. A single
// CTA then reduces the per-cell partials in a fixed order, so every result
// is reproducible from run to run.
#include <algorithm>
#include <cmath>
#include <vector>

#include "eg_internal.h"
#include "eg_setup.h"

namespace eg {
namespace {

constexpr double kPiF = 3.141592653589793238462643383279502884;
constexpr int kFineMax = 16;  // points per direction of the fine rule (13 for k <= 8)

// The fine rule in one direction and the Lagrange basis of the q
// Gauss-Legendre nodes at its points (L_i(x_a) at lag[a*q + i]).
struct FineRule1D {
  int nf, q;
  double x[kFineMax], w[kFineMax];
  double lag[kFineMax * EG_MAX_Q];
};

// Cell data shared by every kernel of this file.
struct FieldGeo {
  int nx, ny, n;
  double lx, ly, hx, hy, area, gamma, cos_a, sin_a;
};

enum FieldMode : int { kInitial = 0, kErrors = 1, kDifferences = 2, kIntegral = 3 };

// EulerGas::exact (src/physics.cpp:64-93): the left-going characteristic map
// solved by a safeguarded Newton iteration for the phase of the wave.
__device__ void exact_wave(const FieldGeo &g, double x, double y, double time, double out[4]) {
  const double gm1 = g.gamma - 1.;
  const double drift = (3. - g.gamma) / 2., amplitude = (g.gamma + 1.) / 4.;
  double phase = g.cos_a * x + g.sin_a * y;
  phase -= 2 * floor((phase + 1) / 2);
  phase -= time * drift;
  phase -= 2 * floor((phase + 1) / 2);
  double lo = phase - time * amplitude, hi = phase + time * amplitude, z = phase;
  for (int i = 0; i < 80; i++) {
    const double r = z + time * amplitude * sin(kPiF * z) - phase;
    if (fabs(r) < 2e-15) break;
    if (r > 0)
      hi = z;
    else
      lo = z;
    const double q = z - r / (1 + time * amplitude * kPiF * cos(kPiF * z));
    z = (q >= lo && q <= hi) ? q : .5 * (lo + hi);
  }
  const double jm = sin(kPiF * z), v = 1 + .5 * jm;
  const double sound = gm1 * (2. - jm) / 4.;
  const double rho = pow(sound * sound / g.gamma, 1. / gm1);
  const double pressure = pow(rho, g.gamma);
  out[0] = rho;
  out[1] = rho * v * g.cos_a;
  out[2] = rho * v * g.sin_a;
  out[3] = pressure / gm1 + .5 * rho * v * v;
}

// Lower-left corner of cell e: the element-centre transform of the shifted
// Cartesian mesh minus half a cell (src/problem.cpp:48-72).
__device__ void cell_origin(const FieldGeo &g, int e, double &ox, double &oy) {
  const int ix = e % g.nx, iy = e / g.nx;
  const double x0 = g.lx * ix / g.nx - .5 * g.lx, x1 = g.lx * (ix + 1) / g.nx - .5 * g.lx;
  const double y0 = g.ly * iy / g.ny - .5 * g.ly, y1 = g.ly * (iy + 1) / g.ny - .5 * g.ly;
  const double cx = x0 * .25 + x1 * .25 + x1 * .25 + x0 * .25;
  const double cy = y0 * .25 + y0 * .25 + y1 * .25 + y1 * .25;
  ox = cx - .5 * g.hx;
  oy = cy - .5 * g.hy;
}

// MODE kInitial: out_u <- the L2 projection of the exact wave at `time`.
// MODE kErrors / kDifferences: partial[4e + c] <- the cell's integral of
// (u_h - exact)^2 or (u_h - v_h)^2, component c. MODE kIntegral:
// partial[4e + c] <- the cell's integral of u_h (collocated weights).
template <int Q, int MODE>
__global__ void __launch_bounds__(256)
    field_cell_kernel(FieldGeo g, FineRule1D fr, double time, const double *__restrict__ tab,
                      const double *__restrict__ u, const double *__restrict__ v, double *__restrict__ out_u,
                      double *__restrict__ partial) {
  constexpr int P = Q * Q, M = 4 * P;
  __shared__ double vq[kFineMax * kFineMax][4];
  __shared__ double ue[M];
  const int nf = fr.nf, nq = nf * nf;
  const double *w = tab + TabLayout<Q>::W, *inv_mass = tab + TabLayout<Q>::IM;
  for (int e = blockIdx.x; e < g.n; e += gridDim.x) {
    __syncthreads();
    if (MODE == kIntegral) {
      if (threadIdx.x < 4) {
        const int c = threadIdx.x;
        double a = 0.;
        for (int i = 0; i < P; ++i) a += g.area * w[i] * u[(size_t)e * M + 4 * i + c];
        partial[4 * (size_t)e + c] = a;
      }
      continue;
    }
    double ox, oy;
    cell_origin(g, e, ox, oy);
    if (MODE != kInitial)
      for (int i = threadIdx.x; i < M; i += blockDim.x)
        ue[i] = MODE == kDifferences ? u[(size_t)e * M + i] - v[(size_t)e * M + i] : u[(size_t)e * M + i];
    if (MODE != kDifferences)
      for (int t = threadIdx.x; t < nq; t += blockDim.x) {
        const int ax = t % nf, ay = t / nf;
        exact_wave(g, ox + g.hx * fr.x[ax], oy + g.hy * fr.x[ay], time, vq[t]);
      }
    __syncthreads();
    if (MODE == kInitial) {
      // each output node sums the points in the reference's order
      for (int o = threadIdx.x; o < M; o += blockDim.x) {
        const int i = o >> 2, c = o & 3, ix = i % Q, iy = i / Q;
        double s = 0.;
        for (int ay = 0; ay < nf; ++ay) {
          const double ly = fr.lag[ay * Q + iy], wy = fr.w[ay];
          for (int ax = 0; ax < nf; ++ax) {
            const double sh = fr.lag[ax * Q + ix] * ly;
            s += fr.w[ax] * wy * sh * vq[ay * nf + ax][c];
          }
        }
        out_u[(size_t)e * M + o] = s * inv_mass[i];
      }
    } else {
      // one thread per point: the discrete solution (or difference) there
      for (int t = threadIdx.x; t < nq; t += blockDim.x) {
        const int ax = t % nf, ay = t / nf;
        double z[4] = {0., 0., 0., 0.};
        for (int iy = 0; iy < Q; ++iy) {
          const double ly = fr.lag[ay * Q + iy];
          for (int ix = 0; ix < Q; ++ix) {
            const double sh = fr.lag[ax * Q + ix] * ly;
            const int i = iy * Q + ix;
#pragma unroll
            for (int c = 0; c < 4; ++c) z[c] += sh * ue[4 * i + c];
          }
        }
        const double wq = fr.w[ax] * fr.w[ay];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const double d = MODE == kErrors ? z[c] - vq[t][c] : z[c];
          vq[t][c] = g.area * wq * d * d;  // this thread's own point only
        }
      }
      __syncthreads();
      if (threadIdx.x < 4) {
        const int c = threadIdx.x;
        double a = 0.;
        for (int t = 0; t < nq; ++t) a += vq[t][c];
        partial[4 * (size_t)e + c] = a;
      }
    }
  }
}

// out[c] = sum over cells of partial[4e + c], in a fixed order (one CTA of
// 256 threads).
__global__ void __launch_bounds__(256) field_reduce_kernel(int n, const double *__restrict__ partial,
                                                           double *__restrict__ out) {
  __shared__ double red[256][4];
  double a[4] = {0., 0., 0., 0.};
  for (int e = threadIdx.x; e < n; e += blockDim.x)
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] += partial[4 * (size_t)e + c];
#pragma unroll
  for (int c = 0; c < 4; ++c) red[threadIdx.x][c] = a[c];
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[threadIdx.x][c] += red[threadIdx.x + k][c];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = red[0][threadIdx.x];
}

FieldGeo field_geo(const Ctx &c) {
  const eg_desc &d = c.desc;
  return FieldGeo{d.nx, d.ny, c.n, d.lx, d.ly, d.hx, d.hy, d.area, d.gamma, std::cos(d.alpha), std::sin(d.alpha)};
}

// The square rule of order max(24, 2k+8) as a tensor of its 1-D rule (the
// Gauss-Legendre points and weights on [0, 1]), with the Lagrange basis of
// the element's nodes at those points.
FineRule1D fine_rule(const eg_desc &d) {
  const int order = std::max(24, 2 * d.k + 8);
  const int nf = (order | 1) / 2 + 1;
  if (nf > kFineMax) fail(EG_ERR_INVALID, "fine quadrature rule too large");
  std::vector<double> x, w;
  host::gauss_legendre(nf, x, w);
  FineRule1D r{};
  r.nf = nf;
  r.q = d.k + 1;
  std::vector<double> nodes(d.ex, d.ex + r.q);
  for (int a = 0; a < nf; ++a) {
    r.x[a] = x[a];
    r.w[a] = w[a];
    for (int i = 0; i < r.q; ++i) r.lag[a * r.q + i] = host::lagrange(nodes, i, x[a]);
  }
  return r;
}

void check_time(const eg_desc &d, double time) {
  const double amplitude = (d.gamma + 1.) / 4.;
  if (!(time >= 0 && time * kPiF * amplitude < 1))
    fail(EG_ERR_STEP_INTERVAL, "Exact solution requires T < 4/((gamma+1)*pi)");
}

template <int MODE>
void launch_field(Ctx &c, double time, const double *u, const double *v, double *out_u) {
  if (!c.field_partial) c.field_partial = c.alloc_n<double>((size_t)4 * c.n + 4);
  const FieldGeo g = field_geo(c);
  const FineRule1D fr = fine_rule(c.desc);
  const int grid = std::min(c.n, 148 * 8);
  ProfScope ps(c, EG_K_VECTOR, MODE == kInitial ? 1 : 2);
  EG_DISPATCH_Q(c.q, (field_cell_kernel<Q, MODE><<<grid, 256, 0, c.stream>>>(g, fr, time, c.tab, u, v, out_u,
                                                                              c.field_partial)));
  EG_CUDA(cudaGetLastError());
  if (MODE != kInitial) {
    field_reduce_kernel<<<1, 256, 0, c.stream>>>(c.n, c.field_partial, c.field_partial + 4 * (size_t)c.n);
    EG_CUDA(cudaGetLastError());
  }
}

void fetch4(Ctx &c, double out[4], bool root) {
  EG_CUDA(cudaMemcpyAsync(c.hscal, c.field_partial + 4 * (size_t)c.n, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                          c.stream));
  c.sync();
  for (int k = 0; k < 4; ++k) out[k] = root ? std::sqrt(c.hscal[k]) : c.hscal[k];
}

}  // namespace

void field_initial(Ctx &c, double *u) { launch_field<kInitial>(c, 0., nullptr, nullptr, u); }

void field_errors(Ctx &c, const double *u, double time, double out[4]) {
  check_time(c.desc, time);
  launch_field<kErrors>(c, time, u, nullptr, nullptr);
  fetch4(c, out, true);
}

void field_integral(Ctx &c, const double *u, double out[4]) {
  launch_field<kIntegral>(c, 0., u, nullptr, nullptr);
  fetch4(c, out, false);
}

void field_differences(Ctx &c, const double *u, const double *v, double out[4]) {
  launch_field<kDifferences>(c, 0., u, v, nullptr);
  fetch4(c, out, true);
}

}  // namespace eg
