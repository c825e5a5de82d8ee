// Block ILU(0) preconditioner on the DG cell graph or the condensed HDG face
// graph, natural ordering (FixedBlockILU, src/block_ilu.cpp:10-109;
// Problem::SolverGraph, src/block_ilu.cpp:110-124).
//
// Structure (host, once per context and form): BSR rows in natural order with
// sorted block columns, the diagonal entry of each row, and for every
// strictly lower entry (i,k) the (target i,j ; upper k,j) products that ILU(0)
// retains (block_ilu.cpp:46-57).
//
// Numeric fill (every refresh): DG blocks are the cell Jacobian blocks and the
// face couplings of PartialDGOperator::FillBlocks (src/partial.cpp:140-170);
// HDG blocks are D - sum over cells of the panels C_s X_{s,o}
// (ElementOperator::FillBlocks, src/operators.cpp:48-74), summed in cell order.
//
// Factor and apply are dependency-driven sweeps, one cooperative launch each.
// Rows are grouped in chunks of one grid row (2nx faces or nx cells); chunk c
// belongs to CTA c mod G, and every CTA walks its rows in increasing
// (forward, factor) or decreasing (backward) order. A CTA publishes how many
// of its rows are final in one 64-bit counter tagged with the launch's epoch;
// a row waits only for rows earlier in the sweep order, which co-resident
// CTAs own, so no wait can depend on itself. Every wait is bounded in time
// (IluPlan::wait_limit_ns, far above the longest legitimate wait, which a
// whole factor or sweep bounds): on timeout the kernel records
// DERR_WAIT_LIMIT, sets the abort word, and all CTAs leave at their next wait
// (after their own bulk copies have landed).
//
// The factor stores the explicit inverse of each factored diagonal block
// (pivoted LU applied to the identity), so RightSolve becomes a product with
// it and the backward solve a block GEMV; the arithmetic is the reference's up
// to rounding.
#include <algorithm>
#include <vector>

#include "eg_bulk.cuh"
#include "eg_cellmat.cuh"
#include "eg_internal.h"

namespace eg {
namespace {

constexpr unsigned kCopySpinLimit = 1u << 16;   // try_wait itself suspends between polls
constexpr unsigned kDrainSpinLimit = 1u << 24;  // abort path: let an issued copy land
constexpr int kStageBlocks = 4;             // blocks staged per warp and row
constexpr int kStageMaxB = 36;              // larger blocks are read from global memory
constexpr size_t kSweepSmemBudget = 210 * 1024;
constexpr size_t kRingBytes = 48 * 1024;    // shared-memory ring of finished rows per CTA

// ------------------------------------------------------------ sync helpers
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *)p; }

__device__ __forceinline__ void give_up(int *abort, int *err) {
  atomicExch(abort, 1);
  raise_err(err, DERR_WAIT_LIMIT);
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits are bounded in time: a wait that has polled for more than limit_ns
// nanoseconds (read every 64 polls from the global timer) gives up.
// Bounded wait until *p >= target (another CTA's progress).
__device__ bool wait_progress(const unsigned long long *p, unsigned long long target, int *abort, int *err,
                              unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (ld_acquire(p) >= target) return true;
    if (ld_volatile(abort)) return false;
    if (it >= 16) __nanosleep(64);
    if ((it & 63u) == 0) {
      const unsigned long long now = global_ns();
      if (it == 0) t0 = now;
      else if (now - t0 > limit_ns) break;
    }
  }
  give_up(abort, err);
  return false;
}
// Bounded wait until the CTA's own published row count reaches target.
__device__ bool wait_local(const volatile unsigned *count, unsigned target, int *abort, int *err,
                           unsigned long long limit_ns) {
  unsigned long long t0 = 0;
  for (unsigned it = 0;; ++it) {
    if (*count >= target) return true;
    if (ld_volatile(abort)) return false;
    if (it >= 16) __nanosleep(32);
    if ((it & 63u) == 0) {
      const unsigned long long now = global_ns();
      if (it == 0) t0 = now;
      else if (now - t0 > limit_ns) break;
    }
  }
  give_up(abort, err);
  return false;
}
// The progress value a wait needs: `starve` (a test setting) asks for one no
// CTA ever publishes, so every wait on another CTA runs out.
__device__ __forceinline__ unsigned long long need(unsigned long long tag, int slot, int starve) {
  return starve ? ~0ull : (tag | (unsigned long long)(slot + 1));
}

// ------------------------------------------------------------- scheduling
// Rows of one sweep, host-built for a fixed grid G: chunk c (one grid row of
// faces or cells) belongs to CTA c mod G, whose slots walk its rows in
// increasing (forward, factor) or decreasing (backward) order. For every
// slot the table holds (row, first entry, entry count) and, for each entry
// the sweep reads, its producer (owner CTA << 22 | owner slot) and row.
constexpr int kMaxDeps = 8;
constexpr int kOwnerShift = 22;
constexpr int kSlotMask = (1 << kOwnerShift) - 1;

__device__ __forceinline__ void publish_max(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.max.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ------------------------------------------------------------ sweep kernel
struct SweepArgs {
  int B, ring;
  const int *slot_ptr;
  const int4 *meta;
  const int2 *deps;
  const double *data, *dinv;
  const double *in;  // forward: b; backward: the forward result w
  double *out;       // forward: w; backward: x
  unsigned long long *progress;
  int *abort, *err;
  unsigned long long tag;
  int staged;        // stage up to kStageBlocks blocks per row in shared memory
  unsigned long long limit_ns;  // bound of every wait
  int starve;        // test setting: waits on other CTAs can never be met
};

// FixedBlockILU::Mult (src/block_ilu.cpp:88-109). Forward: w_i = b_i -
// sum_{j<i} L_ij w_j. Backward: x_i = U_ii^{-1} (w_i - sum_{j>i} U_ij x_j).
// One warp per row (lanes own block rows r = lane + 32 s); the W warps of a
// CTA keep W rows and their block copies in flight. A finished row goes to a
// shared-memory ring (read by later rows of the same CTA) and to global
// memory; the CTA's own count is published first, then, off the local chain,
// the release of the global counter that other CTAs poll.
template <int S, bool BACK>
__global__ void __launch_bounds__(256, 1) ilu_sweep_kernel(SweepArgs a) {
  extern __shared__ __align__(128) double smem[];
  __shared__ unsigned done_local;
  __shared__ __align__(8) unsigned long long bars[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, W = blockDim.x >> 5;
  const int g = blockIdx.x, B = a.B;
  const size_t BB = (size_t)B * B;
  const int p0 = a.slot_ptr[g], nslots = a.slot_ptr[g + 1] - p0;
  const size_t stage_doubles = a.staged ? kStageBlocks * BB : 0;
  double *stage = smem + (size_t)warp * stage_doubles;
  double *vb = smem + (size_t)W * stage_doubles + (size_t)warp * 32 * S;
  double *ring = smem + (size_t)W * (stage_doubles + 32 * S);
  if (threadIdx.x == 0) done_local = 0;
  if (a.staged && lane == 0) mbar_init(&bars[warp]);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  volatile unsigned *dl = &done_local;
  unsigned phase = 0;
  int4 nm = make_int4(0, 0, 0, 0);
  int2 nd[kMaxDeps];
  auto fetch = [&](int slot) {
    if (slot < nslots) {
      nm = a.meta[p0 + slot];
#pragma unroll
      for (int k = 0; k < kMaxDeps; ++k) nd[k] = a.deps[(size_t)(p0 + slot) * kMaxDeps + k];
    }
  };
  fetch(warp);
  for (int slot = warp; slot < nslots; slot += W) {
    const int i = nm.x, e0 = nm.y, ne = nm.z;
    int2 dep[kMaxDeps];
#pragma unroll
    for (int k = 0; k < kMaxDeps; ++k) dep[k] = nd[k];
    fetch(slot + W);  // the next row's schedule is in flight during this row
    const int nst = a.staged ? min(ne, BACK ? kStageBlocks - 1 : kStageBlocks) : 0;
    const bool copy = a.staged && (nst > 0 || BACK);
    if (copy && lane == 0) {
      const unsigned bytes = (unsigned)(sizeof(double) * BB * (nst + (BACK ? 1 : 0)));
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect(&bars[warp], bytes);
      if (nst) bulk_load(stage, a.data + (size_t)e0 * BB, (unsigned)(sizeof(double) * BB * nst), &bars[warp]);
      if (BACK) bulk_load(stage + (size_t)nst * BB, a.dinv + (size_t)i * BB, (unsigned)(sizeof(double) * BB),
                          &bars[warp]);
    }
    double acc[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int r = lane + 32 * s;
      acc[s] = r < B ? __ldcg(a.in + (size_t)i * B + r) : 0.;
    }
    if (copy) {
      if (!mbar_wait(&bars[warp], phase, kCopySpinLimit)) {
        give_up(a.abort, a.err);
        // let the copy land before the CTA can exit; if even the longer drain
        // bound runs out, the copy may still write this CTA's shared memory:
        // err[2] tells the host that the context can no longer be trusted
        if (!mbar_wait(&bars[warp], phase, kDrainSpinLimit) && lane == 0) atomicExch(a.err + 2, 1);
        return;
      }
      phase ^= 1u;
    }
    bool ok = true;
#pragma unroll
    for (int k = 0; k < kMaxDeps; ++k) {
      if (k < ne && ok) {
        const int owner = dep[k].x >> kOwnerShift, js = dep[k].x & kSlotMask, j = dep[k].y;
        const bool local = owner == g;
        ok = local ? wait_local(dl, (unsigned)js + 1, a.abort, a.err, a.limit_ns)
                   : wait_progress(a.progress + owner, need(a.tag, js, a.starve), a.abort, a.err, a.limit_ns);
        if (ok) {
          __threadfence_block();
          const bool in_ring = local && slot - js <= a.ring - W;
          const double *src = ring + (size_t)(js & (a.ring - 1)) * B;
          for (int r = lane; r < B; r += 32) vb[r] = in_ring ? src[r] : __ldcg(a.out + (size_t)j * B + r);
          __syncwarp();
          const double *A = k < nst ? stage + (size_t)k * BB : a.data + (size_t)(e0 + k) * BB;
#pragma unroll
          for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            if (r < B) {
              double t = acc[s];
              for (int cc = 0; cc < B; ++cc) t -= A[(size_t)cc * B + r] * vb[cc];
              acc[s] = t;
            }
          }
          __syncwarp();
        }
      }
    }
    if (!ok) return;
    if (BACK) {
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const int r = lane + 32 * s;
        if (r < B) vb[r] = acc[s];
      }
      __syncwarp();
      const double *Di = a.staged ? stage + (size_t)nst * BB : a.dinv + (size_t)i * BB;
#pragma unroll
      for (int s = 0; s < S; ++s) {
        const int r = lane + 32 * s;
        if (r < B) {
          double t = 0.;
          for (int cc = 0; cc < B; ++cc) t += Di[(size_t)cc * B + r] * vb[cc];
          acc[s] = t;
        }
      }
      __syncwarp();
    }
    double *rs = ring + (size_t)(slot & (a.ring - 1)) * B;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int r = lane + 32 * s;
      if (r < B) {
        a.out[(size_t)i * B + r] = acc[s];
        rs[r] = acc[s];
      }
    }
    __threadfence_block();
    __syncwarp();
    int pub = 1;
    if (lane == 0) {
      pub = wait_local(dl, (unsigned)slot, a.abort, a.err, a.limit_ns);  // rows are published in order
      if (pub) {
        *dl = (unsigned)slot + 1;
        publish_max(a.progress + g, a.tag | (unsigned long long)(slot + 1));
      }
    }
    if (!__shfl_sync(0xffffffffu, pub, 0)) return;
  }
}

// ----------------------------------------------------------- factor kernel
struct FactorArgs {
  int B, maxrow, maxupd;
  const int *slot_ptr;
  const int4 *meta;   // forward schedule: (row, first lower entry, lower count)
  const int2 *deps;
  const int *row, *diag, *upd_ptr, *upd;
  double *data, *dinv, *work;
  unsigned long long *progress;
  int *abort, *err;
  unsigned long long tag;
  unsigned long long limit_ns;  // bound of every wait
  int starve;                   // test setting: waits on other CTAs can never be met
};

// FixedBlockILU::Factor (src/block_ilu.cpp:74-87), one CTA per row: for each
// lower entry (i,k) in column order, L_ik = A_ik U_kk^{-1}, then A_ij -= L_ik
// U_kj over the retained products; finally the pivoted LU of the diagonal
// block, stored as its explicit inverse. With SMEM the row's blocks, U_kk^{-1}
// and the U_kj of one step are staged in shared memory.
template <int RMAX, bool SMEM>
__global__ void __launch_bounds__(256, 1) ilu_factor_kernel(FactorArgs a) {
  extern __shared__ __align__(16) double fsm[];
  __shared__ int piv_s[32 * RMAX];
  __shared__ double inv_piv[32 * RMAX];
  __shared__ double bcast[2];
  __shared__ int stop;
  const int B = a.B;
  const int BB = B * B;
  const int g = blockIdx.x, p0 = a.slot_ptr[g], nslots = a.slot_ptr[g + 1] - p0;
  double *Lt, *Sd, *Inv, *rowblk = nullptr, *Dk = nullptr, *Ub = nullptr;
  if (SMEM) {
    rowblk = fsm;                         // the row's blocks (maxrow)
    Dk = rowblk + (size_t)a.maxrow * BB;  // U_kk^{-1}
    Ub = Dk + BB;                         // the U_kj of one step (maxupd)
    Lt = Ub + (size_t)a.maxupd * BB;
  } else {
    Lt = a.work + (size_t)g * 3 * BB;
  }
  Sd = Lt + BB;
  Inv = Sd + BB;
  for (int slot = 0; slot < nslots; ++slot) {
    const int4 m = a.meta[p0 + slot];
    const int i = m.x, rb = a.row[i], re = a.row[i + 1], di = a.diag[i];
    if (threadIdx.x == 0) {
      int ok = 1;
      for (int k = 0; k < m.z && ok; ++k) {
        const int2 d = a.deps[(size_t)(p0 + slot) * kMaxDeps + k];
        const int owner = d.x >> kOwnerShift, js = d.x & kSlotMask;
        if (owner != g)
          ok = wait_progress(a.progress + owner, need(a.tag, js, a.starve), a.abort, a.err, a.limit_ns);
      }
      stop = !ok;
    }
    if (SMEM)
      for (int o = threadIdx.x; o < (re - rb) * BB; o += blockDim.x) rowblk[o] = a.data[(size_t)rb * BB + o];
    __syncthreads();
    if (stop) return;
    for (int ik = rb; ik < di; ++ik) {
      const int kk = a.deps[(size_t)(p0 + slot) * kMaxDeps + (ik - rb)].y;
      const int u0 = a.upd_ptr[ik], nu = a.upd_ptr[ik + 1] - u0;
      double *Aik = SMEM ? rowblk + (size_t)(ik - rb) * BB : a.data + (size_t)ik * BB;
      const double *Dsrc = a.dinv + (size_t)kk * BB;
      if (SMEM) {
        for (int o = threadIdx.x; o < BB; o += blockDim.x) Dk[o] = __ldcg(Dsrc + o);
        for (int t = threadIdx.x; t < nu * BB; t += blockDim.x)
          Ub[t] = __ldcg(a.data + (size_t)a.upd[2 * (u0 + t / BB) + 1] * BB + t % BB);
        __syncthreads();
      }
      for (int o = threadIdx.x; o < BB; o += blockDim.x) {
        const int r = o % B, cc = o / B;
        double sum = 0.;
        if (SMEM) {
          for (int s = 0; s < B; ++s) sum += Aik[(size_t)s * B + r] * Dk[(size_t)cc * B + s];
        } else {
          for (int s = 0; s < B; ++s) sum += Aik[(size_t)s * B + r] * __ldcg(Dsrc + (size_t)cc * B + s);
        }
        Lt[o] = sum;
      }
      __syncthreads();
      for (int o = threadIdx.x; o < BB; o += blockDim.x) Aik[o] = Lt[o];
      for (int t = threadIdx.x; t < nu * BB; t += blockDim.x) {
        const int uu = t / BB, o = t % BB;
        const int r = o % B, cc = o / B;
        const int target = a.upd[2 * (u0 + uu)];
        double *T = SMEM ? rowblk + (size_t)(target - rb) * BB : a.data + (size_t)target * BB;
        double sum = 0.;
        if (SMEM) {
          const double *U = Ub + (size_t)uu * BB;
          for (int s = 0; s < B; ++s) sum += Lt[(size_t)s * B + r] * U[(size_t)cc * B + s];
        } else {
          const double *U = a.data + (size_t)a.upd[2 * (u0 + uu) + 1] * BB;
          for (int s = 0; s < B; ++s) sum += Lt[(size_t)s * B + r] * __ldcg(U + (size_t)cc * B + s);
        }
        T[o] -= sum;
      }
      __syncthreads();
    }
    const double *Ad = SMEM ? rowblk + (size_t)(di - rb) * BB : a.data + (size_t)di * BB;
    for (int o = threadIdx.x; o < BB; o += blockDim.x) {
      Sd[o] = Ad[o];
      Inv[o] = (o % B) == (o / B) ? 1. : 0.;
    }
    __syncthreads();
    const bool ok = cta_lu_solve<RMAX>(Sd, B, Inv, B, B, B, piv_s, inv_piv, bcast);
    if (!ok && threadIdx.x == 0) raise_err(a.err, DERR_SINGULAR_ILU);
    double *Di = a.dinv + (size_t)i * BB;
    for (int o = threadIdx.x; o < BB; o += blockDim.x) Di[o] = Inv[o];
    if (SMEM)
      for (int o = threadIdx.x; o < (re - rb) * BB; o += blockDim.x) a.data[(size_t)rb * BB + o] = rowblk[o];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) publish_max(a.progress + g, a.tag | (unsigned long long)(slot + 1));
  }
}

// ------------------------------------------------------------ fill kernels
// HDG: all 16 panels C_s R_s X_{:,o} of every cell (FaceCoupling::Panel,
// src/operators.cpp:7-26), layout [cell][s][o][t x t column-major].
template <int Q>
__global__ void __launch_bounds__(256)
    ilu_panels_kernel(Geo g, const double *__restrict__ tab, const double *__restrict__ XY,
                      const double *__restrict__ Cb, double *__restrict__ panels16) {
  constexpr int P = Q * Q, M = 4 * P, T = 4 * Q, NR = 4 * T + 1, TT = T * T;
  __shared__ STab<Q> st;
  load_tables<Q>(st, tab);
  __syncthreads();
  const long long total = (long long)g.n * 16 * TT;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(o / (16 * TT)), rem = (int)(o % (16 * TT));
    const int pan = rem / TT, r2 = rem % TT;
    const int row = r2 % T, cc = r2 / T;
    const int s = pan >> 2, so = pan & 3, jj = row >> 2, c = row & 3;
    const double *xc = XY + (size_t)e * M * NR + (size_t)(so * T + cc) * M;
    double val[4] = {0., 0., 0., 0.};
    for (int l = 0; l < Q; ++l) {
      const double f = st.fb(s, jj, l);
      const double *xv = xc + 4 * line_node<Q>(s, jj, l);
#pragma unroll
      for (int d = 0; d < 4; ++d) val[d] += f * xv[d];
    }
    const double *cb = Cb + ((size_t)e * 4 * Q + s * Q + jj) * 16;
    double res = 0.;
#pragma unroll
    for (int d = 0; d < 4; ++d) res += cb[c + 4 * d] * val[d];
    panels16[o] = res;
  }
}

// HDG block (f, g) = delta_fg D_f - sum over cells holding both faces of the
// cell's panel (side of f, side of g), in cell order (operators.cpp:48-74).
__global__ void __launch_bounds__(256)
    ilu_fill_hdg_kernel(int nnzb, int T, const int *__restrict__ erow, const int *__restrict__ col,
                        const int *__restrict__ fill_ptr, const int *__restrict__ fill_src,
                        const double *__restrict__ D, const double *__restrict__ panels16,
                        double *__restrict__ data) {
  const int TT = T * T;
  const long long total = (long long)nnzb * TT;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(o / TT), r2 = (int)(o % TT);
    const int row = r2 % T, cc = r2 / T;
    const int f = erow[b];
    double v = (f == col[b] && row == cc) ? D[(size_t)f * T + row] : 0.;
    for (int p = fill_ptr[b]; p < fill_ptr[b + 1]; ++p) v = v - panels16[(size_t)fill_src[p] * TT + r2];
    data[o] = v;
  }
}

// DG blocks (PartialDGOperator::FillBlocks, src/partial.cpp:140-170): the
// diagonal is the cell block of block Jacobi; an off-diagonal block (a, b)
// holds, for every face joining a and b (in face order), +scale M^-1 phi phi jr
// when a is the face's left cell and -scale M^-1 phi phi jl when it is the
// right one. One CTA per block.
template <int Q>
__global__ void __launch_bounds__(256)
    ilu_fill_dg_kernel(Geo g, const double *__restrict__ tab, Frozen fz, const double *__restrict__ u,
                       int nnzb, const int *__restrict__ erow, const int *__restrict__ col,
                       const int *__restrict__ fill_ptr, const int *__restrict__ fill_src, double *data) {
  constexpr int P = Q * Q, M = 4 * P;
  __shared__ STab<Q> st;
  __shared__ double us[M], UT[16 * Q], FM[4 * Q * 16];
  load_tables<Q>(st, tab);
  for (int b = blockIdx.x; b < nnzb; b += gridDim.x) {
    __syncthreads();
    const int ea = erow[b], eb = col[b];
    double *A = data + (size_t)b * M * M;
    if (ea == eb) {
      for (int i = threadIdx.x; i < M; i += blockDim.x) us[i] = u[(size_t)ea * M + i];
      __syncthreads();
      cell_traces<Q>(st, us, UT);
      __syncthreads();
      dg_face_matrices<Q>(UT, FM, g, fz, ea);
      __syncthreads();
      build_cell_matrix<Q>(A, M, st, us, FM, g);
      continue;
    }
    for (int o = threadIdx.x; o < M * M; o += blockDim.x) A[o] = 0.;
    __syncthreads();
    for (int p = fill_ptr[b]; p < fill_ptr[b + 1]; ++p) {
      const int code = fill_src[p];
      const int f = code >> 1;
      const bool right = (code & 1) != 0;  // block row cell is the face's right cell
      const int L = f >> 1, axis = f & 1, ls = axis ? 3 : 1, rs = ls - 1;
      const int R = neighbour(L, ls, g.nx, g.ny);
      const int ts = right ? rs : ls, trs = right ? ls : rs, tc = right ? L : R;
      const double len = axis ? g.hx : g.hy;
      for (int j = threadIdx.x; j < Q; j += blockDim.x) {
        double tr[4], jm[16];
        trace4<Q>(st, u, tc, trs, j, tr);
        jacobian(tr, axis, g.gm1, jm);
        const int fi = f * Q + j;
        const double wgt = right ? fz.lw[fi] : fz.rw[fi], pen = right ? fz.pen[fi] : -fz.pen[fi];
#pragma unroll
        for (int k = 0; k < 16; ++k) FM[j * 16 + k] = wgt * jm[k] + ((k % 5) == 0 ? pen : 0.);
      }
      __syncthreads();
      for (int t = threadIdx.x; t < Q * Q * Q * 16; t += blockDim.x) {
        const int j = t / (Q * Q * 16), rem = t % (Q * Q * 16);
        const int li = rem / (Q * 16), lk = (rem / 16) % Q, cd = rem % 16, c = cd & 3, d = cd >> 2;
        const int i = line_node<Q>(ts, j, li), kk = line_node<Q>(trs, j, lk);
        const double scale = g.dt * len / g.area * st.ew(j);
        const double w = (right ? -scale : scale) * st.inv_mass(i) * st.fb(ts, j, li) * st.fb(trs, j, lk);
        A[(size_t)(4 * kk + d) * M + 4 * i + c] += w * FM[j * 16 + c + 4 * d];
      }
      __syncthreads();
    }
  }
}

int sm_count_ilu() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// ------------------------------------------------------------ host: plan
template <class Kern>
int per_sm(Kern kern, int block, size_t smem) {
  // the opt-in covers dynamic sizes whose sum with the static shared memory passes 48 KB
  if (smem > 0) EG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int n = 0;
  EG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, block, smem));
  return n;
}

template <int S>
int sweep_occupancy(int block, size_t smem) {
  return std::min(per_sm(ilu_sweep_kernel<S, false>, block, smem), per_sm(ilu_sweep_kernel<S, true>, block, smem));
}
int sweep_occupancy_dispatch(int S, int block, size_t smem) {
  switch (S) {
    case 1: return sweep_occupancy<1>(block, smem);
    case 2: return sweep_occupancy<2>(block, smem);
    case 3: return sweep_occupancy<3>(block, smem);
    case 4: return sweep_occupancy<4>(block, smem);
    case 5: return sweep_occupancy<5>(block, smem);
    case 6: return sweep_occupancy<6>(block, smem);
    case 7: return sweep_occupancy<7>(block, smem);
    case 8: return sweep_occupancy<8>(block, smem);
    case 9: return sweep_occupancy<9>(block, smem);
    case 10: return sweep_occupancy<10>(block, smem);
    case 11: return sweep_occupancy<11>(block, smem);
    default: fail(EG_ERR_INVALID, "unsupported block size");
  }
}
int factor_occupancy(int B, bool staged, size_t smem) {
  if (staged)
    return B <= 32 ? per_sm(ilu_factor_kernel<1, true>, 256, smem) : per_sm(ilu_factor_kernel<2, true>, 256, smem);
  switch ((B + 31) / 32) {
    case 2: return per_sm(ilu_factor_kernel<2, false>, 256, 0);
    case 3: return per_sm(ilu_factor_kernel<3, false>, 256, 0);
    case 4: return per_sm(ilu_factor_kernel<4, false>, 256, 0);
    case 5: return per_sm(ilu_factor_kernel<5, false>, 256, 0);
    case 6: return per_sm(ilu_factor_kernel<6, false>, 256, 0);
    case 7: return per_sm(ilu_factor_kernel<7, false>, 256, 0);
    case 8: return per_sm(ilu_factor_kernel<8, false>, 256, 0);
    case 9: return per_sm(ilu_factor_kernel<9, false>, 256, 0);
    case 10: return per_sm(ilu_factor_kernel<10, false>, 256, 0);
    case 11: return per_sm(ilu_factor_kernel<11, false>, 256, 0);
    default: fail(EG_ERR_INVALID, "unsupported block size");
  }
}

void build_plan(Ctx &c, int form) {
  IluPlan &P = c.ilu[form];
  if (P.built) return;
  const bool hdg = form == EG_FORM_HDG;
  const int nx = c.desc.nx, ny = c.desc.ny;
  P.rows = hdg ? c.nf : c.n;
  P.B = hdg ? c.t : c.m;
  P.chunk = hdg ? 2 * nx : nx;
  P.chunks = ny;
  // Problem::SolverGraph (src/block_ilu.cpp:110-124) plus the row itself
  std::vector<std::vector<int>> graph(P.rows);
  if (hdg) {
    for (int e = 0; e < c.n; ++e)
      for (int s = 0; s < 4; ++s)
        for (int o = 0; o < 4; ++o) graph[cell_face(e, s, nx, ny)].push_back(cell_face(e, o, nx, ny));
  } else {
    for (int e = 0; e < c.n; ++e) graph[e].push_back(e);
    for (int f = 0; f < c.nf; ++f) {
      const int L = f >> 1, R = neighbour(L, (f & 1) ? 3 : 1, nx, ny);
      graph[L].push_back(R);
      graph[R].push_back(L);
    }
  }
  std::vector<int> row(1, 0), col, diag(P.rows), erow;
  for (int i = 0; i < P.rows; ++i) {
    auto &r = graph[i];
    r.push_back(i);
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    for (int j : r) {
      if (j == i) diag[i] = (int)col.size();
      col.push_back(j);
      erow.push_back(i);
    }
    row.push_back((int)col.size());
  }
  P.nnzb = (int)col.size();
  // retained ILU(0) products (src/block_ilu.cpp:46-57)
  std::vector<int> upd_ptr(1, 0), upd;
  P.maxupd = 1;
  for (int i = 0; i < P.rows; ++i) {
    for (int ik = row[i]; ik < row[i + 1]; ++ik) {
      int count = 0;
      if (ik < diag[i]) {
        const int k = col[ik];
        int ij = ik + 1, kj = diag[k] + 1;
        while (ij < row[i + 1] && kj < row[k + 1]) {
          if (col[ij] < col[kj]) {
            ++ij;
          } else if (col[kj] < col[ij]) {
            ++kj;
          } else {
            upd.push_back(ij);
            upd.push_back(kj);
            ++count;
            ++ij;
            ++kj;
          }
        }
      }
      P.maxupd = std::max(P.maxupd, count);
      upd_ptr.push_back((int)upd.size() / 2);
    }
  }
  auto at = [&](int i, int j) {
    const auto it = std::lower_bound(col.begin() + row[i], col.begin() + row[i + 1], j);
    return (int)(it - col.begin());
  };
  // fill contributions per entry
  std::vector<std::vector<int>> contrib(P.nnzb);
  if (hdg) {
    for (int e = 0; e < c.n; ++e)
      for (int s = 0; s < 4; ++s)
        for (int o = 0; o < 4; ++o)
          contrib[at(cell_face(e, s, nx, ny), cell_face(e, o, nx, ny))].push_back(e * 16 + s * 4 + o);
  } else {
    for (int f = 0; f < c.nf; ++f) {
      const int L = f >> 1, R = neighbour(L, (f & 1) ? 3 : 1, nx, ny);
      contrib[at(L, R)].push_back(2 * f);
      contrib[at(R, L)].push_back(2 * f + 1);
    }
  }
  std::vector<int> fill_ptr(1, 0), fill_src;
  for (auto &v : contrib) {
    fill_src.insert(fill_src.end(), v.begin(), v.end());
    fill_ptr.push_back((int)fill_src.size());
  }
  if (fill_src.empty()) fill_src.push_back(0);
  if (upd.empty()) upd.push_back(0);
  P.maxl = P.maxu = P.maxrow = 0;
  for (int i = 0; i < P.rows; ++i) {
    P.maxl = std::max(P.maxl, diag[i] - row[i]);
    P.maxu = std::max(P.maxu, row[i + 1] - diag[i] - 1);
    P.maxrow = std::max(P.maxrow, row[i + 1] - row[i]);
  }
  if (P.maxl > kMaxDeps || P.maxu > kMaxDeps) fail(EG_ERR_INVALID, "block ILU row too long");
  // launch shapes; every CTA of a sweep must be resident (cooperative launch)
  const int sms = sm_count_ilu();
  const size_t BB = (size_t)P.B * P.B;
  const int S = (P.B + 31) / 32;
  P.staged = P.B <= kStageMaxB ? 1 : 0;
  P.ring = 1;
  while ((size_t)(2 * P.ring) * P.B * sizeof(double) <= kRingBytes) P.ring *= 2;
  int W = 8;
  auto sweep_smem = [&](int w) {
    return sizeof(double) * ((size_t)w * (P.staged ? kStageBlocks * BB : 0) + (size_t)w * 32 * S +
                             (size_t)P.ring * P.B);
  };
  while (W > 1 && sweep_smem(W) > kSweepSmemBudget) --W;
  if (P.ring < 2 * W) fail(EG_ERR_INVALID, "block ILU ring too small");
  P.sweep_warps = W;
  P.sweep_smem = sweep_smem(W);
  P.factor_smem = P.staged ? sizeof(double) * BB * (size_t)(P.maxrow + P.maxupd + 4) : 0;
  const int occ = std::min(sweep_occupancy_dispatch(S, 32 * W, P.sweep_smem),
                           factor_occupancy(P.B, P.staged != 0, P.factor_smem));
  if (occ < 1) fail(EG_ERR_INVALID, "block ILU kernels do not fit on an SM");
  const int G = std::min(P.chunks, std::min(occ, 2) * sms);
  P.grid_sweep = P.grid_factor = G;
  // schedules (the forward one is also the factor's)
  auto upload = [&](const std::vector<int> &v) {
    int *d = c.alloc_n<int>(v.size());
    EG_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, c.stream));
    c.sync();  // the host vector is local
    return d;
  };
  for (int back = 0; back < 2; ++back) {
    std::vector<int> slot_ptr(G + 1, 0), owner_of(P.rows), slot_of(P.rows);
    std::vector<std::vector<int>> rows_of(G);
    for (int g = 0; g < G; ++g) {
      std::vector<int> chunks;
      for (int ch = g; ch < P.chunks; ch += G) chunks.push_back(ch);
      if (back) std::reverse(chunks.begin(), chunks.end());
      for (int ch : chunks)
        for (int o = 0; o < P.chunk; ++o) {
          const int i = ch * P.chunk + (back ? P.chunk - 1 - o : o);
          owner_of[i] = g;
          slot_of[i] = (int)rows_of[g].size();
          rows_of[g].push_back(i);
        }
      slot_ptr[g + 1] = slot_ptr[g] + (int)rows_of[g].size();
    }
    if (slot_ptr[G] != P.rows) fail(EG_ERR_INVALID, "block ILU schedule does not cover the rows");
    std::vector<int> meta((size_t)P.rows * 4, 0), deps((size_t)P.rows * kMaxDeps * 2, 0);
    for (int g = 0; g < G; ++g)
      for (size_t s = 0; s < rows_of[g].size(); ++s) {
        const int i = rows_of[g][s];
        const size_t pos = (size_t)slot_ptr[g] + s;
        const int e0 = back ? diag[i] + 1 : row[i], e1 = back ? row[i + 1] : diag[i];
        meta[pos * 4] = i;
        meta[pos * 4 + 1] = e0;
        meta[pos * 4 + 2] = e1 - e0;
        for (int e = e0; e < e1; ++e) {
          const int j = col[e], k = e - e0;
          // a row reads only rows that come earlier in its own CTA's order
          if (owner_of[j] == g && slot_of[j] >= (int)s) fail(EG_ERR_INVALID, "block ILU schedule order");
          if (slot_of[j] > kSlotMask) fail(EG_ERR_INVALID, "block ILU schedule too long");
          deps[(pos * kMaxDeps + k) * 2] = (owner_of[j] << kOwnerShift) | slot_of[j];
          deps[(pos * kMaxDeps + k) * 2 + 1] = j;
        }
      }
    P.slot_ptr[back] = upload(slot_ptr);
    P.meta[back] = upload(meta);
    P.deps[back] = upload(deps);
  }
  P.row = upload(row);
  P.col = upload(col);
  P.diag = upload(diag);
  P.erow = upload(erow);
  P.upd_ptr = upload(upd_ptr);
  P.upd = upload(upd);
  P.fill_ptr = upload(fill_ptr);
  P.fill_src = upload(fill_src);
  P.data = c.alloc_n<double>((size_t)P.nnzb * BB);
  P.dinv = c.alloc_n<double>((size_t)P.rows * BB);
  P.w = c.alloc_n<double>((size_t)P.rows * P.B);
  // the condensation keeps all 16 panels per cell where the Schur action
  // streams them (same layout and arithmetic); otherwise the fill forms them
  if (hdg && c.geo.npan != 16) P.panels16 = c.alloc_n<double>((size_t)c.n * 16 * BB);
  if (!P.staged) P.work = c.alloc_n<double>((size_t)G * 3 * BB);
  P.progress = c.alloc_n<unsigned long long>(G);
  EG_CUDA(cudaMemsetAsync(P.progress, 0, sizeof(unsigned long long) * G, c.stream));
  P.abort = c.alloc_n<int>(1);
  EG_CUDA(cudaMemsetAsync(P.abort, 0, sizeof(int), c.stream));
  P.epoch = 0;
  P.wait_limit_ns = c.ilu_wait_limit_ns;
  P.starve = c.ilu_starve;
  P.built = true;
}

template <class Kern, class Args>
void launch_coop(Kern kern, int grid, int block, size_t smem, cudaStream_t s, Args &args) {
  void *params[] = {&args};
  EG_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), grid, block, params, smem, s));
}

template <int S, bool BACK>
void sweep(Ctx &c, IluPlan &P, const double *in, double *out) {
  SweepArgs a{};
  a.B = P.B;
  a.ring = P.ring;
  a.slot_ptr = P.slot_ptr[BACK];
  a.meta = reinterpret_cast<const int4 *>(P.meta[BACK]);
  a.deps = reinterpret_cast<const int2 *>(P.deps[BACK]);
  a.data = P.data;
  a.dinv = P.dinv;
  a.in = in;
  a.out = out;
  a.progress = P.progress;
  a.abort = P.abort;
  a.err = c.derr;
  a.tag = (unsigned long long)(++P.epoch) << 32;
  a.staged = P.staged;
  a.limit_ns = P.wait_limit_ns;
  a.starve = P.starve;
  launch_coop(ilu_sweep_kernel<S, BACK>, P.grid_sweep, 32 * P.sweep_warps, P.sweep_smem, c.stream, a);
}

template <bool BACK>
void sweep_dispatch(Ctx &c, IluPlan &P, const double *in, double *out) {
  switch ((P.B + 31) / 32) {
    case 1: sweep<1, BACK>(c, P, in, out); break;
    case 2: sweep<2, BACK>(c, P, in, out); break;
    case 3: sweep<3, BACK>(c, P, in, out); break;
    case 4: sweep<4, BACK>(c, P, in, out); break;
    case 5: sweep<5, BACK>(c, P, in, out); break;
    case 6: sweep<6, BACK>(c, P, in, out); break;
    case 7: sweep<7, BACK>(c, P, in, out); break;
    case 8: sweep<8, BACK>(c, P, in, out); break;
    case 9: sweep<9, BACK>(c, P, in, out); break;
    case 10: sweep<10, BACK>(c, P, in, out); break;
    case 11: sweep<11, BACK>(c, P, in, out); break;
    default: fail(EG_ERR_INVALID, "unsupported block size");
  }
}

template <int RMAX, bool SMEM>
void factor_launch(Ctx &c, IluPlan &P) {
  FactorArgs a{};
  a.B = P.B;
  a.maxrow = P.maxrow;
  a.maxupd = P.maxupd;
  a.slot_ptr = P.slot_ptr[0];
  a.meta = reinterpret_cast<const int4 *>(P.meta[0]);
  a.deps = reinterpret_cast<const int2 *>(P.deps[0]);
  a.row = P.row;
  a.diag = P.diag;
  a.upd_ptr = P.upd_ptr;
  a.upd = P.upd;
  a.data = P.data;
  a.dinv = P.dinv;
  a.work = P.work;
  a.progress = P.progress;
  a.abort = P.abort;
  a.err = c.derr;
  a.tag = (unsigned long long)(++P.epoch) << 32;
  a.limit_ns = P.wait_limit_ns;
  a.starve = P.starve;
  launch_coop(ilu_factor_kernel<RMAX, SMEM>, P.grid_factor, 256, SMEM ? P.factor_smem : 0, c.stream, a);
}

void factor_dispatch(Ctx &c, IluPlan &P) {
  if (P.staged) {
    if (P.B <= 32) factor_launch<1, true>(c, P);
    else factor_launch<2, true>(c, P);
    return;
  }
  switch ((P.B + 31) / 32) {
    case 2: factor_launch<2, false>(c, P); break;
    case 3: factor_launch<3, false>(c, P); break;
    case 4: factor_launch<4, false>(c, P); break;
    case 5: factor_launch<5, false>(c, P); break;
    case 6: factor_launch<6, false>(c, P); break;
    case 7: factor_launch<7, false>(c, P); break;
    case 8: factor_launch<8, false>(c, P); break;
    case 9: factor_launch<9, false>(c, P); break;
    case 10: factor_launch<10, false>(c, P); break;
    case 11: factor_launch<11, false>(c, P); break;
    default: fail(EG_ERR_INVALID, "unsupported block size");
  }
}

// Numeric blocks of the plan's structure into dst (nnzb x B^2, column-major).
void fill_blocks(Ctx &c, int form, IluPlan &P, double *dst) {
  const bool hdg = form == EG_FORM_HDG;
  const int sms = sm_count_ilu();
  if (hdg) {
    const double *pan16 = c.geo.npan == 16 ? c.panels : P.panels16;
    if (c.geo.npan != 16) {
      const long long np = (long long)c.n * 16 * c.t * c.t;
      const int grid = (int)std::min<long long>((np + 255) / 256, (long long)sms * 16);
      EG_DISPATCH_Q(c.q, (ilu_panels_kernel<Q><<<grid, 256, 0, c.stream>>>(c.geo, c.tab, c.XY, c.Cb, P.panels16)));
      EG_CUDA(cudaGetLastError());
    }
    const long long ne = (long long)P.nnzb * c.t * c.t;
    const int g2 = (int)std::min<long long>((ne + 255) / 256, (long long)sms * 16);
    ilu_fill_hdg_kernel<<<g2, 256, 0, c.stream>>>(P.nnzb, c.t, P.erow, P.col, P.fill_ptr, P.fill_src, c.D,
                                                  pan16, dst);
  } else {
    const int grid = std::min(P.nnzb, sms * 8);
    EG_DISPATCH_Q(c.q, (ilu_fill_dg_kernel<Q><<<grid, 256, 0, c.stream>>>(
                           c.geo, c.tab, Frozen{c.fa, c.fbb, c.flw, c.frw, c.fpen}, c.u, P.nnzb, P.erow, P.col,
                           P.fill_ptr, P.fill_src, dst)));
  }
  EG_CUDA(cudaGetLastError());
}

// y = A x for an assembled block-sparse operator: one thread per scalar row;
// blocks are column-major, so consecutive rows of a block read adjacent
// entries, and block columns come in increasing order (the column order of
// the assembled CSR rows, src/operators.cpp:180-238).
__global__ void __launch_bounds__(256)
    bsr_spmv_kernel(int rows, int B, const int *__restrict__ rowp, const int *__restrict__ col,
                    const double *__restrict__ data, const double *__restrict__ x, double *__restrict__ y,
                    const int *__restrict__ skip) {
  if (skip != nullptr && *skip) return;  // speculative Arnoldi step after convergence
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (long long)rows * B) return;
  const int i = (int)(id / B), r = (int)(id % B);
  const size_t BB = (size_t)B * B;
  double acc = 0.;
  for (int k = rowp[i]; k < rowp[i + 1]; ++k) {
    const double *a = data + (size_t)k * BB + r;
    const double *xv = x + (size_t)col[k] * B;
#pragma unroll 4
    for (int j = 0; j < B; ++j) acc += a[(size_t)j * B] * xv[j];
  }
  y[id] = acc;
}

}  // namespace

void ilu_refresh(Ctx &c, int form, bool factor) {
  build_plan(c, form);
  IluPlan &P = c.ilu[form];
  const bool hdg = form == EG_FORM_HDG;
  if (hdg && !c.condensed) fail(EG_ERR_INVALID, "Schur preconditioner requires a condensation");
  ProfScope ps(c, hdg ? EG_K_SCHUR_JACOBI : EG_K_DG_JACOBI, factor ? 3 : 2);
  EG_CUDA(cudaMemsetAsync(P.abort, 0, sizeof(int), c.stream));
  fill_blocks(c, form, P, P.data);
  if (factor) factor_dispatch(c, P);
}

// ElementOperator::Assemble (src/operators.cpp:180-238) for full assembly and
// the element-assembled DG Jacobian (Problem::DG, src/problem.cpp:552-588):
// the blocks the ILU(0) fill sums (FillBlocks), left unfactored.
void assemble_blocks(Ctx &c, int form) {
  const bool hdg = form == EG_FORM_HDG;
  if (hdg && !c.condensed) fail(EG_ERR_INVALID, "assembled Schur operator requires a condensation");
  build_plan(c, form);
  IluPlan &P = c.ilu[form];
  ProfScope ps(c, EG_K_VECTOR, 2);
  if (c.opts.precond == EG_PC_BLOCK_ILU0) {
    if (!P.asm_own) P.asm_own = c.alloc_n<double>((size_t)P.nnzb * P.B * P.B);
    P.asmd = P.asm_own;
  } else {
    P.asmd = P.data;  // unused by block Jacobi
  }
  fill_blocks(c, form, P, P.asmd);
}

void launch_assembled_apply(Ctx &c, int form, const double *x, double *y) {
  IluPlan &P = c.ilu[form];
  if (!P.built || !P.asmd) fail(EG_ERR_INVALID, "no assembled operator");
  ProfScope ps(c, form == EG_FORM_HDG ? EG_K_SCHUR_APPLY : EG_K_DG_APPLY, 2);
  const long long total = (long long)P.rows * P.B;
  bsr_spmv_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c.stream>>>(P.rows, P.B, P.row, P.col, P.asmd, x,
                                                                         y, c.skip);
  EG_CUDA(cudaGetLastError());
}

void launch_ilu_apply(Ctx &c, int form, const double *b, double *x) {
  IluPlan &P = c.ilu[form];
  if (!P.built) fail(EG_ERR_INVALID, "no preconditioner built");
  ProfScope ps(c, EG_K_PC_APPLY, 2);
  // a sweep that gave up leaves the abort word set; every apply starts clear
  EG_CUDA(cudaMemsetAsync(P.abort, 0, sizeof(int), c.stream));
  sweep_dispatch<false>(c, P, b, P.w);
  sweep_dispatch<true>(c, P, P.w, x);
}

}  // namespace eg
