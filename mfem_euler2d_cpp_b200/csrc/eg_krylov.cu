// Weighted vector algebra and restarted right-preconditioned CGS2 GMRES
// (LinearSolver::Impl, src/linear.cpp:11-157), resident on the device.
//
// Every reduction runs on a fixed grid of kRedBlocks blocks; each block writes
// its partial sums and the last block to finish adds the partials in block
// order, so results are bitwise reproducible for a given size. The dual-norm
// metric is not stored: it is periodic (cell metric |K| M_ii repeats every m
// entries, trace metric len_f / ew_j every 2t entries) and is read from a
// small table staged in shared memory.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "eg_internal.h"

namespace eg {

__device__ __forceinline__ double block_sum(double v, double *red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// Returns true in the last block to finish (after all partials are visible).
__device__ __forceinline__ bool last_block(unsigned *counter) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned ticket = atomicAdd(counter, 1u);
    is_last = ticket == gridDim.x - 1;
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

constexpr int kChunk = 8;  // Krylov columns per register chunk

// Sum of n CTA partials p[0..n) by one warp in a fixed order: lane l adds
// p[l + 32 i] into four interleaved accumulators (four independent loads in
// flight instead of one dependent chain), then a warp tree. The order depends
// on n only, so the result is bitwise reproducible for a given grid.
__device__ __forceinline__ double warp_sum_partials(const double *__restrict__ p, int n) {
  const int lane = threadIdx.x & 31;
  double t0 = 0., t1 = 0., t2 = 0., t3 = 0.;
  int b = lane;
  for (; b + 96 < n; b += 128) {
    t0 += p[b];
    t1 += p[b + 32];
    t2 += p[b + 64];
    t3 += p[b + 96];
  }
  for (; b < n; b += 32) t0 += p[b];
  double t = (t0 + t1) + (t2 + t3);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
  return t;
}

// ---------------------------------------------------------- weighted norm
template <class T>
__global__ void __launch_bounds__(kRedThreads)
    wnorm2_kernel(int N, const T *__restrict__ x, const double *__restrict__ mtab, int period,
                  double *partials, unsigned *counter, double *out) {
  __shared__ double red[kRedThreads];
  __shared__ double mt[2 * EG_MAX_P];
  for (int i = threadIdx.x; i < period / 4; i += blockDim.x) mt[i] = mtab[i];
  __syncthreads();
  double s = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double v = (double)x[i];
    s += mt[(i % period) >> 2] * v * v;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (last_block(counter)) {
    double t = 0.;
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += partials[b];
    t = block_sum(t, red);
    if (threadIdx.x == 0) {
      *out = t;
      *counter = 0;
    }
  }
}

// Givens update of Hessenberg column j and the convergence test
// (src/linear.cpp:123-136), run by the last CTA of the norm pass once
// h(j+1, j) = next is known: the column and the earlier rotations are staged
// in shared memory by the CTA, thread 0 applies the chain.
__device__ void givens_step(GmresCtl *ctl, int R, int j, double *st /* 3 * (kMaxRestart + 1) */) {
  const int ld = R + 1;
  double *hc = st, *cs = st + (kMaxRestart + 1), *sn = cs + (kMaxRestart + 1);
  for (int i = threadIdx.x; i <= j + 1; i += blockDim.x) hc[i] = ctl->h[i + ld * j];
  for (int i = threadIdx.x; i < j; i += blockDim.x) {
    cs[i] = ctl->cs[i];
    sn[i] = ctl->sn[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < j; ++i) {
      const double u = hc[i], v = hc[i + 1];
      hc[i] = cs[i] * u + sn[i] * v;
      hc[i + 1] = -sn[i] * u + cs[i] * v;
    }
    const double d = hypot(hc[j], hc[j + 1]);
    if (!(isfinite(d) && d > 0)) {
      ctl->err = 1;
      ctl->stop = 1;
    } else {
      const double c = hc[j] / d, s = hc[j + 1] / d;
      hc[j] = d;
      hc[j + 1] = 0.;
      const double gj = ctl->g[j];
      ctl->cs[j] = c;
      ctl->sn[j] = s;
      ctl->g[j + 1] = -s * gj;
      ctl->g[j] = c * gj;
      ctl->count = j + 1;
      ctl->stop = (fabs(ctl->g[j + 1]) <= ctl->abs_tol || ctl->next <= DBL_MIN) ? 1 : 0;
      ctl->j = j + 1;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= j + 1; i += blockDim.x) ctl->h[i + ld * j] = hc[i];
}

// ------------------------------------------------------------ CGS2 passes
// MODE 0: proj = V^T (metric w)                        (first pass)
// MODE 1: w -= V proj_in; proj = V^T (metric w)        (second pass)
// MODE 2: w -= V proj_in; next = ||w||_metric         (norm)
// proj results are added into the Hessenberg column (h(i,j) += proj_i).
// T is the storage type of the Krylov vectors; sums are formed in FP64.
template <int MODE, class T>
__global__ void __launch_bounds__(kRedThreads)
    cgs_kernel(int N, T *__restrict__ w, const T *__restrict__ V, size_t ldv, int ncols,
               const double *__restrict__ mtab, int period, double *partials, unsigned *counter,
               GmresCtl *ctl, int R) {
  __shared__ double red[kRedThreads];
  __shared__ double mt[2 * EG_MAX_P];
  __shared__ double pin[kMaxRestart + 1];
  if (ctl->stop) return;  // speculative Arnoldi step after convergence
  for (int i = threadIdx.x; i < period / 4; i += blockDim.x) mt[i] = mtab[i];
  if (MODE > 0)
    for (int i = threadIdx.x; i < ncols; i += blockDim.x) pin[i] = ctl->proj[i];
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  const int j = ctl->j;
  if (MODE == 2) {
    double s = 0.;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
      double comb = 0.;
      for (int c = 0; c < ncols; ++c) comb += (double)V[c * ldv + i] * pin[c];
      const T v = (T)((double)w[i] - comb);
      w[i] = v;
      s += mt[(i % period) >> 2] * (double)v * (double)v;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
    if (last_block(counter)) {
      double t = 0.;
      for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += partials[b];
      t = block_sum(t, red);
      if (threadIdx.x == 0) {
        const double next = sqrt(t);
        ctl->next = next;
        ctl->inv_next = next > 0 ? 1. / next : 0.;
        ctl->h[(j + 1) + (R + 1) * j] = next;
        *counter = 0;
      }
      __syncthreads();
      givens_step(ctl, R, j, red);
    }
    return;
  }
  if (MODE == 1) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
      double comb = 0.;
      for (int c = 0; c < ncols; ++c) comb += (double)V[c * ldv + i] * pin[c];
      w[i] = (T)((double)w[i] - comb);
    }
    // each thread re-reads only its own elements below: no grid barrier needed
  }
  for (int c0 = 0; c0 < ncols; c0 += kChunk) {
    const int nc = min(kChunk, ncols - c0);
    double acc[kChunk];
#pragma unroll
    for (int k = 0; k < kChunk; ++k) acc[k] = 0.;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
      const double wm = mt[(i % period) >> 2] * (double)w[i];
#pragma unroll
      for (int k = 0; k < kChunk; ++k)
        if (k < nc) acc[k] += (double)V[(c0 + k) * ldv + i] * wm;
    }
    for (int k = 0; k < nc; ++k) {
      const double s = block_sum(acc[k], red);
      if (threadIdx.x == 0) partials[(size_t)(c0 + k) * gridDim.x + blockIdx.x] = s;
    }
  }
  if (last_block(counter)) {
    for (int c = 0; c < ncols; ++c) {
      double t = 0.;
      for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += partials[(size_t)c * gridDim.x + b];
      t = block_sum(t, red);
      if (threadIdx.x == 0) {
        ctl->proj[c] = t;
        ctl->h[c + (R + 1) * j] += t;
      }
    }
    if (threadIdx.x == 0) *counter = 0;
  }
}

// Register-resident CGS2 passes for up to NC basis columns: every element's
// basis values are loaded once per pass and reused for the update of w and
// the projection, each thread keeps several elements' loads in flight, and
// sums are reduced with warp shuffles, then across the CTA, then in block
// order by the last CTA (fixed grid: bitwise reproducible). Same MODE
// semantics as cgs_kernel.
constexpr int kCgsBlocks = 592;  // 4 CTAs per SM
constexpr int kCgsThreads = 256;
static_assert(kCgsBlocks * 24 <= kRedBlocks * (kMaxRestart + 1), "partials hold every CTA's column sums");
// Grid of the register CGS passes for a vector of length N: about four
// elements per thread, at most kCgsBlocks CTAs (a function of N only, so the
// summation order stays fixed for a given problem).
inline int cgs_grid(int N) { return std::max(1, std::min(kCgsBlocks, (N + 4 * kCgsThreads - 1) / (4 * kCgsThreads))); }

template <int NC>
__device__ __forceinline__ void cta_reduce_columns(double (&acc)[NC], int nc, double *red /* [8][NC] */,
                                                   double *partials, int nblocks) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    double v = acc[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0 && k < nc) red[warp * NC + k] = v;
  }
  __syncthreads();
  if (threadIdx.x < nc) {
    double t = 0.;
    for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) t += red[wv * NC + threadIdx.x];
    partials[(size_t)threadIdx.x * nblocks + blockIdx.x] = t;
  }
}

template <int MODE, class T, int NC>
__global__ void __launch_bounds__(kCgsThreads)
    cgs_reg_kernel(int N, T *__restrict__ w, const T *__restrict__ V, size_t ldv, int ncols,
                   const double *__restrict__ mtab, int period, double *partials, unsigned *counter,
                   GmresCtl *ctl, int R) {
  __shared__ double red[8 * NC];
  __shared__ double mt[2 * EG_MAX_P];
  __shared__ double pin[NC];
  __shared__ double gst[MODE == 2 ? 3 * (kMaxRestart + 1) : 1];  // Givens staging (norm pass)
  // the control words, the metric and the projections are independent loads:
  // issue them together and test for a stopped cycle after (a speculative
  // Arnoldi step after convergence returns without touching w)
  const int stop = ctl->stop, j = ctl->j;
  for (int i = threadIdx.x; i < period / 4; i += blockDim.x) mt[i] = mtab[i];
  if (MODE > 0)
    for (int i = threadIdx.x; i < ncols; i += blockDim.x) pin[i] = ctl->proj[i];
  if (stop) return;
  __syncthreads();
  double acc[NC];
#pragma unroll
  for (int k = 0; k < NC; ++k) acc[k] = 0.;
  const int stride = gridDim.x * blockDim.x;
  // U elements a stride apart per iteration, their loads issued together
  // (same per-thread order of elements as one at a time)
  constexpr int U = (sizeof(T) == 8 && NC <= 16) ? 2 : 1;  // FP64 vectors (measured)
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < N; i0 += U * stride) {
    double v[U][NC], wv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int iu = i0 + u * stride;
      const int ic = iu < N ? iu : i0;
#pragma unroll
      for (int k = 0; k < NC; ++k) v[u][k] = k < ncols ? (double)V[(size_t)k * ldv + ic] : 0.;
      wv[u] = (double)w[ic];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * stride;
      if (i < N) {
        const double m = mt[(i % period) >> 2];
        double wi = wv[u];
        if (MODE > 0) {
          double comb = 0.;
#pragma unroll
          for (int k = 0; k < NC; ++k) comb += v[u][k] * (k < ncols ? pin[k] : 0.);
          const T wn = (T)(wi - comb);
          w[i] = wn;
          wi = (double)wn;
        }
        if (MODE == 2) {
          acc[0] += m * wi * wi;
        } else {
          const double wm = m * wi;
#pragma unroll
          for (int k = 0; k < NC; ++k) acc[k] += v[u][k] * wm;
        }
      }
    }
  }
  const int nred = MODE == 2 ? 1 : ncols;
  cta_reduce_columns<NC>(acc, nred, red, partials, gridDim.x);
  if (last_block(counter)) {
    // one warp per column (warp_sum_partials: fixed order, bitwise reproducible)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < nred; c += kCgsThreads / 32) {
      const double t = warp_sum_partials(partials + (size_t)c * gridDim.x, (int)gridDim.x);
      if (lane == 0) {
        if (MODE == 2) {
          const double next = sqrt(t);
          ctl->next = next;
          ctl->inv_next = next > 0 ? 1. / next : 0.;
          ctl->h[(j + 1) + (R + 1) * j] = next;
        } else {
          ctl->proj[c] = t;
          ctl->h[c + (R + 1) * j] += t;
        }
      }
    }
    if (MODE == 2) {
      __syncthreads();  // next and h(j+1, j) written by thread 0
      givens_step(ctl, R, j, gst);
    }
    if (threadIdx.x == 0) *counter = 0;
  }
}

// V_{j+1} = w * (1/next) when next > 0 (src/linear.cpp:119-122)
template <class T>
__global__ void normalize_kernel(int N, const T *__restrict__ w, T *__restrict__ vnext, const GmresCtl *ctl) {
  const double next = ctl->next;
  const int stop = ctl->stop;
  if (!(next > 0) || stop) return;  // a stopped cycle never reads V_{j+1}
  const double s = 1. / next;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    vnext[i] = (T)((double)w[i] * s);
}

// Upper-triangular solve for the Krylov coefficients (src/linear.cpp:138-142).
__global__ void backsub_kernel(GmresCtl *ctl, int R) {
  const int count = ctl->count, ld = R + 1;
  for (int i = count - 1; i >= 0; --i) {
    double v = ctl->g[i];
    for (int k = i + 1; k < count; ++k) v -= ctl->h[i + ld * k] * ctl->y[k];
    ctl->y[i] = v / ctl->h[i + ld * i];
  }
}

__global__ void cycle_init_kernel(GmresCtl *ctl, int R, double beta, double abs_tol) {
  for (int i = threadIdx.x; i < (R + 1) * R; i += blockDim.x) ctl->h[i] = 0.;
  for (int i = threadIdx.x; i <= R; i += blockDim.x) ctl->g[i] = 0.;
  __syncthreads();
  if (threadIdx.x == 0) {
    ctl->g[0] = beta;
    ctl->j = 0;
    ctl->count = 0;
    ctl->stop = 0;
    ctl->err = 0;
    ctl->abs_tol = abs_tol;
  }
}

// out = V[:, 0:count] y (src/linear.cpp:145-146)
template <class T>
__global__ void combine_kernel(int N, const T *__restrict__ V, size_t ldv, const GmresCtl *__restrict__ ctl,
                               T *__restrict__ out) {
  __shared__ double ys[kMaxRestart];
  const int count = ctl->count;
  for (int i = threadIdx.x; i < count; i += blockDim.x) ys[i] = ctl->y[i];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    double s = 0.;
    for (int c = 0; c < count; ++c) s += (double)V[c * ldv + i] * ys[c];
    out[i] = (T)s;
  }
}

__global__ void axpby_kernel(int N, double a, const double *__restrict__ x, double b,
                             const double *__restrict__ y, double *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i];
}
template <class T>
__global__ void scale_kernel(int N, double a, const T *__restrict__ x, T *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    out[i] = (T)((double)x[i] * a);
}
template <class T>
__global__ void sub_kernel(int N, const T *__restrict__ x, const T *__restrict__ y, T *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    out[i] = x[i] - y[i];
}
template <class T>
__global__ void add_kernel(int N, const T *__restrict__ x, T *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    y[i] += x[i];
}
template <class T>
__global__ void fill_kernel(int N, T v, T *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) out[i] = v;
}

static int vec_grid(int N) { return std::max(1, std::min((N + 255) / 256, 148 * 16)); }

template <class T>
void launch_wnorm2_t(Ctx &c, const T *x, int N, const double *mtab, int period, int slot) {
  ProfScope ps(c, EG_K_KRYLOV, 1);
  // a grid that depends on N only keeps the summation order fixed per problem
  const int grid = std::max(1, std::min(kRedBlocks, (N + 4 * kRedThreads - 1) / (4 * kRedThreads)));
  wnorm2_kernel<T><<<grid, kRedThreads, 0, c.stream>>>(N, x, mtab, period, c.partials, c.counter, c.dscal + slot);
  EG_CUDA(cudaGetLastError());
}
void launch_wnorm2(Ctx &c, const double *x, int N, const double *mtab, int period, int slot) {
  launch_wnorm2_t(c, x, N, mtab, period, slot);
}
template <class T>
double wnorm_t(Ctx &c, const T *x, int N, const double *mtab, int period) {
  launch_wnorm2_t(c, x, N, mtab, period, DS_NORM);
  EG_CUDA(cudaMemcpyAsync(c.hscal + DS_NORM, c.dscal + DS_NORM, sizeof(double),
                          cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return std::sqrt(c.hscal[DS_NORM]);
}
double wnorm(Ctx &c, const double *x, int N, const double *mtab, int period) {
  launch_wnorm2(c, x, N, mtab, period, DS_NORM);
  EG_CUDA(cudaMemcpyAsync(c.hscal + DS_NORM, c.dscal + DS_NORM, sizeof(double),
                          cudaMemcpyDeviceToHost, c.stream));
  c.sync();
  return std::sqrt(c.hscal[DS_NORM]);
}
double cell_norm(Ctx &c, const double *x) { return wnorm(c, x, c.nu, c.mtab_dg, c.m); }

void launch_axpby(Ctx &c, int N, double a, const double *x, double b, const double *y, double *out) {
  ProfScope ps(c, EG_K_VECTOR, 1);
  axpby_kernel<<<vec_grid(N), 256, 0, c.stream>>>(N, a, x, b, y, out);
  EG_CUDA(cudaGetLastError());
}
void launch_copy(Ctx &c, int N, const double *x, double *out) {
  if (x != out)
    EG_CUDA(cudaMemcpyAsync(out, x, sizeof(double) * N, cudaMemcpyDeviceToDevice, c.stream));
}
void launch_fill(Ctx &c, int N, double v, double *out) {
  ProfScope ps(c, EG_K_VECTOR, 1);
  fill_kernel<double><<<vec_grid(N), 256, 0, c.stream>>>(N, v, out);
  EG_CUDA(cudaGetLastError());
}

// CTAs of KERN (kCgsThreads each) resident at once on the device: one wave.
// Queried once per kernel; a property of the kernel and the device only.
template <auto KERN>
int cgs_wave() {
  static const int wave = [] {
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, KERN, kCgsThreads, 0) != cudaSuccess) per_sm = 1;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
    cudaGetLastError();
    return std::max(1, per_sm) * std::max(1, sms);
  }();
  return wave;
}

// The three CGS2 passes of Arnoldi step j (src/linear.cpp:104-118).
template <class T, int NC>
void cgs_reg_passes(Ctx &c, int N, T *w, const T *V, size_t ldv, int nc, const double *mtab, int period, int R) {
  // each pass at most one wave of resident CTAs (the passes differ in
  // registers); the grid depends on N and the device only, so the summation
  // order stays fixed
  const int g0 = std::min(cgs_grid(N), cgs_wave<cgs_reg_kernel<0, T, NC>>());
  const int g1 = std::min(cgs_grid(N), cgs_wave<cgs_reg_kernel<1, T, NC>>());
  const int g2 = std::min(cgs_grid(N), cgs_wave<cgs_reg_kernel<2, T, NC>>());
  cgs_reg_kernel<0, T, NC><<<g0, kCgsThreads, 0, c.stream>>>(N, w, V, ldv, nc, mtab, period, c.partials,
                                                                   c.counter, c.ctl, R);
  cgs_reg_kernel<1, T, NC><<<g1, kCgsThreads, 0, c.stream>>>(N, w, V, ldv, nc, mtab, period, c.partials,
                                                                   c.counter, c.ctl, R);
  cgs_reg_kernel<2, T, NC><<<g2, kCgsThreads, 0, c.stream>>>(N, w, V, ldv, nc, mtab, period, c.partials,
                                                                   c.counter, c.ctl, R);
}
template <class T>
void cgs_passes(Ctx &c, int N, T *w, const T *V, size_t ldv, int nc, const double *mtab, int period, int R) {
  if (nc <= 4) {
    cgs_reg_passes<T, 4>(c, N, w, V, ldv, nc, mtab, period, R);
  } else if (nc <= 8) {
    cgs_reg_passes<T, 8>(c, N, w, V, ldv, nc, mtab, period, R);
  } else if (nc <= 16) {
    cgs_reg_passes<T, 16>(c, N, w, V, ldv, nc, mtab, period, R);
  } else if (nc <= 24) {
    cgs_reg_passes<T, 24>(c, N, w, V, ldv, nc, mtab, period, R);
  } else {
    cgs_kernel<0, T><<<kRedBlocks, kRedThreads, 0, c.stream>>>(N, w, V, ldv, nc, mtab, period, c.partials,
                                                               c.counter, c.ctl, R);
    cgs_kernel<1, T><<<kRedBlocks, kRedThreads, 0, c.stream>>>(N, w, V, ldv, nc, mtab, period, c.partials,
                                                               c.counter, c.ctl, R);
    cgs_kernel<2, T><<<kRedBlocks, kRedThreads, 0, c.stream>>>(N, w, V, ldv, nc, mtab, period, c.partials,
                                                               c.counter, c.ctl, R);
  }
}

// -------------------------------------------------------------------- GMRES
// Weighted restarted CGS2 GMRES on vectors of type T (FP64 for the parity
// path, FP32 for the inner solve of mixed precision); scalars, Hessenberg,
// Givens and all sums are FP64.
template <class T>
double gmres_t(Ctx &c, LinearOpsT<T> &ops, const KrylovBufs<T> &kb, const T *rhs, T *x, double tol, int limit,
               bool zero_guess, bool require_converged, int *count, double *rhs_norm_out,
               double known_rhs_norm) {
  const int N = ops.N;
  const int R = std::min(N, kb.R);
  const size_t ldv = kb.ld;
  T *res = kb.res, *w = kb.w, *z = kb.z, *V = kb.V;
  if (zero_guess) {
    {
      ProfScope ps(c, EG_K_VECTOR, 1);
      fill_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, T(0), x);
      EG_CUDA(cudaGetLastError());
    }
    EG_CUDA(cudaMemcpyAsync(res, rhs, sizeof(T) * N, cudaMemcpyDeviceToDevice, c.stream));
  } else {
    ops.apply(c, x, w);
    ProfScope ps(c, EG_K_VECTOR, 1);
    sub_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, rhs, w, res);
    EG_CUDA(cudaGetLastError());
  }
  const double rhs_norm = known_rhs_norm >= 0. ? known_rhs_norm : wnorm_t(c, rhs, N, ops.mtab, ops.period);
  if (rhs_norm_out) *rhs_norm_out = rhs_norm;
  *count = 0;
  if (rhs_norm == 0.) return 0.;
  int iterations = 0;
  // from a zero guess the residual is a copy of rhs: the same reduction result
  double residual_norm = zero_guess ? rhs_norm : wnorm_t(c, res, N, ops.mtab, ops.period);
  while (iterations < limit) {
    const double beta = residual_norm;
    if (beta <= tol * rhs_norm) break;
    {
      ProfScope ps(c, EG_K_KRYLOV, 2);
      scale_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, 1 / beta, res, V);
      cycle_init_kernel<<<1, 256, 0, c.stream>>>(c.ctl, R, beta, tol * rhs_norm);
      EG_CUDA(cudaGetLastError());
    }
    // Arnoldi steps are enqueued in groups of ops.group with one host check
    // of the device stop flag per group; the steps of a group that follow the
    // converged one return at once (Ctx::skip, and the stop check of the CGS
    // and normalisation kernels), so iterates and counts are those of a
    // check after every step.
    for (int j = 0; j < R && iterations < limit;) {
      const int group = std::max(1, std::min(ops.group, std::min(R - j, limit - iterations)));
      struct SkipGuard {
        Ctx &c;
        ~SkipGuard() { c.skip = nullptr; }
      } guard{c};
      c.skip = group > 1 ? &c.ctl->stop : nullptr;
      for (int b = 0; b < group; ++b) {
        const int jj = j + b;
        const T *vj = V + (size_t)jj * ldv;
        ops.precondition(c, vj, z);
        ops.apply(c, z, w);
        ProfScope ps(c, EG_K_KRYLOV, 4);
        cgs_passes<T>(c, N, w, V, ldv, jj + 1, ops.mtab, ops.period, R);
        normalize_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, w, V + (size_t)(jj + 1) * ldv, c.ctl);
        EG_CUDA(cudaGetLastError());
      }
      c.skip = nullptr;
      // j, count, stop and err of the control block
      EG_CUDA(cudaMemcpyAsync(&c.hctl->j, &c.ctl->j, 4 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      if (c.hctl->err) fail(EG_ERR_GMRES_BREAKDOWN, "GMRES Arnoldi breakdown");
      const int done = c.hctl->count - j;  // steps completed in this group
      iterations += done;
      j += done;
      if (c.hctl->stop || done < group) break;
    }
    {
      ProfScope ps(c, EG_K_KRYLOV, 2);
      backsub_kernel<<<1, 1, 0, c.stream>>>(c.ctl, R);
      combine_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, V, ldv, c.ctl, kb.comb);
      EG_CUDA(cudaGetLastError());
    }
    ops.precondition(c, kb.comb, kb.corr);
    {
      ProfScope ps(c, EG_K_VECTOR, 1);
      add_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, kb.corr, x);
    }
    ops.apply(c, x, w);
    {
      ProfScope ps(c, EG_K_VECTOR, 1);
      sub_kernel<T><<<vec_grid(N), 256, 0, c.stream>>>(N, rhs, w, res);
      EG_CUDA(cudaGetLastError());
    }
    residual_norm = wnorm_t(c, res, N, ops.mtab, ops.period);
    if (!std::isfinite(residual_norm)) fail(EG_ERR_GMRES_NONFINITE, "Nonfinite GMRES residual");
  }
  *count = iterations;
  if (require_converged && !(residual_norm <= tol * rhs_norm))
    fail(EG_ERR_GMRES_LIMIT, "GMRES iteration limit reached");
  return residual_norm;
}

double gmres(Ctx &c, LinearOps &ops, const double *rhs, double *x, double tol, int limit,
             bool zero_guess, int *count, double *rhs_norm_out, double known_rhs_norm) {
  c.ensure_krylov();
  // columns of the operator's own length, contiguous
  const KrylovBufs<double> kb{c.V, c.kw, c.kz, c.kres, c.kcomb, c.kcorr, (size_t)ops.N, c.kR};
  return gmres_t<double>(c, ops, kb, rhs, x, tol, limit, zero_guess, true, count, rhs_norm_out, known_rhs_norm);
}

double gmres_f32(Ctx &c, LinearOpsT<float> &ops, const KrylovBufs<float> &kb, const float *rhs, float *x,
                 double tol, int limit, int *count) {
  return gmres_t<float>(c, ops, kb, rhs, x, tol, limit, true, false, count, nullptr, -1.);
}

}  // namespace eg
