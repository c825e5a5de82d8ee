// Allocation-free cell norm: the weighted dual norm of a body vector for
// callers that may not allocate device memory (see eg_cell_norm_noalloc in
// include/euler2d_cuda.h). Its scratch is the static array below; this file
// is the only place that names it.
#include <cmath>
#include <mutex>

#include "eg_internal.h"

namespace {

constexpr int kBlocks = 296;                // fixed reduction grid (deterministic order)
constexpr int kThreads = 256;
constexpr int kMetricOff = 0;               // metric table: EG_MAX_P doubles
constexpr int kPartialOff = EG_MAX_P;       // one partial sum per block
constexpr int kResultOff = kPartialOff + kBlocks;
constexpr int kCounterOff = kResultOff + 1; // completion counter (unsigned, in a double slot)
constexpr int kScratchDoubles = kCounterOff + 1;
static_assert(kScratchDoubles * sizeof(double) <= 4096, "scratch must stay within 4 KB");

// Scratch shared by every call on a device; kept from call to call.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kThreads)
    noalloc_wnorm2_kernel(long long n, const double *__restrict__ x, int period, double *scratch) {
  __shared__ double red[kThreads];
  __shared__ double mt[EG_MAX_P];
  __shared__ bool is_last;
  for (int i = threadIdx.x; i < period / 4; i += blockDim.x) mt[i] = scratch[kMetricOff + i];
  __syncthreads();
  double s = 0.;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i];
    s += mt[(i % period) >> 2] * v * v;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  unsigned *counter = reinterpret_cast<unsigned *>(scratch + kCounterOff);
  if (threadIdx.x == 0) {
    scratch[kPartialOff + blockIdx.x] = red[0];
    __threadfence();
    is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double t = 0.;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t += scratch[kPartialOff + b];
  red[threadIdx.x] = t;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    scratch[kResultOff] = red[0];
    *counter = 0u;
  }
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current).
int scratch_address(double **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return EG_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return EG_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_ptr[dev];
  return EG_OK;
}

}  // namespace

extern "C" int eg_cell_norm_noalloc(const eg_desc *d, const double *r, void *stream, double *out) {
  if (!d || !r || !out) return EG_ERR_INVALID;
  if (d->k < 0 || d->k > EG_MAX_Q - 1 || d->nx < 2 || d->ny < 2) return EG_ERR_INVALID;
  const int q = d->k + 1, p = q * q, m = 4 * p;
  if (p > EG_MAX_P) return EG_ERR_INVALID;  // metric table capacity of the scratch
  // the same descriptor checks as eg_create: lexicographic nodes, a positive cell area
  if (!(d->area > 0.)) return EG_ERR_INVALID;
  for (int i = 0; i < p; ++i)
    if (d->tensor_node[i] != i) return EG_ERR_INVALID;
  const long long n = (long long)d->nx * d->ny * m;
  // the vector must be device-accessible memory: a host pointer would fault the kernel
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, r) != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_INVALID;
  }
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) return EG_ERR_INVALID;
  double *scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != EG_OK) return rc;
  // device memory of another GPU is not reachable without peer access: refuse it
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_CUDA;
  }
  if (attr.type == cudaMemoryTypeDevice && attr.device != dev) return EG_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double table[EG_MAX_P];
  for (int i = 0; i < p; ++i) table[i] = d->area * d->mass[i];
  // the metric table and the completion counter are rewritten by every call
  if (cudaMemcpyAsync(scratch + kMetricOff, table, sizeof(double) * p, cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemsetAsync(scratch + kCounterOff, 0, sizeof(double), s) != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_CUDA;
  }
  noalloc_wnorm2_kernel<<<kBlocks, kThreads, 0, s>>>(n, r, m, scratch);
  double sum = 0.;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&sum, scratch + kResultOff, sizeof(double), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return EG_ERR_CUDA;
  }
  *out = std::sqrt(sum);
  return EG_OK;
}
