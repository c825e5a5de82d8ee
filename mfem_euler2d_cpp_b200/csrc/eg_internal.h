// Host-side context of one problem instance and the kernel launchers shared
// between translation units. Not part of the public C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/euler2d_cuda.h"
#include "eg_device.cuh"

#define EG_DISPATCH_Q(qv, ...)                   \
  switch (qv) {                                  \
    case 1: { constexpr int Q = 1; __VA_ARGS__; } break; \
    case 2: { constexpr int Q = 2; __VA_ARGS__; } break; \
    case 3: { constexpr int Q = 3; __VA_ARGS__; } break; \
    case 4: { constexpr int Q = 4; __VA_ARGS__; } break; \
    case 5: { constexpr int Q = 5; __VA_ARGS__; } break; \
    case 6: { constexpr int Q = 6; __VA_ARGS__; } break; \
    case 7: { constexpr int Q = 7; __VA_ARGS__; } break; \
    case 8: { constexpr int Q = 8; __VA_ARGS__; } break; \
    case 9: { constexpr int Q = 9; __VA_ARGS__; } break; \
    default: break;                              \
  }

namespace eg {

// Thrown inside the library only; converted to a status at the C-ABI.
struct Failure {
  int status;
  std::string msg;
};
[[noreturn]] void fail(int status, const std::string &msg);
void cuda_check(cudaError_t e, const char *what);
#define EG_CUDA(call) ::eg::cuda_check((call), #call)

// Fixed grid of the deterministic reductions (partials are summed in block
// order by the last block to finish).
constexpr int kRedBlocks = 296;
constexpr int kRedThreads = 256;

// Device scalar slots (doubles) used by reductions and control.
enum DScal : int {
  DS_NORM = 0,       // generic reduction result
  DS_NORM2 = 1,
  DS_WAVE = 2,       // max HLL speed bits (as unsigned long long)
  DS_ADMISSIBLE = 3, // 1.0 when admissible
  DS_COUNT = 8
};

// GMRES control block (device). Sized for restart R <= kMaxRestart.
constexpr int kMaxRestart = 64;
struct GmresCtl {
  double h[(kMaxRestart + 1) * kMaxRestart];  // column-major (R+1) x R
  double g[kMaxRestart + 1];
  double cs[kMaxRestart], sn[kMaxRestart], y[kMaxRestart];
  double proj[kMaxRestart + 1];
  double next;         // norm of the orthogonalised Krylov vector
  double inv_next;
  double rhs_norm, tol, abs_tol;
  int j, count, stop, err;
};

struct Ctx;

// Event-timed kernel classes (profiling) and launch counting.
struct Profiler {
  bool on = false;
  struct Rec {
    int id;
    long long launches;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> pool;
  std::vector<Rec> pending;
  double ms[EG_K_COUNT] = {};
  long long count[EG_K_COUNT] = {};
};
// RAII bracket of the launches of one kernel class on the context stream.
struct ProfScope {
  Ctx &c;
  int id;
  long long launches;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(Ctx &ctx, int kernel_class, long long nlaunch);
  ~ProfScope();
};

// Operators used by the Krylov solver, on vectors of type T.
template <class T>
struct LinearOpsT {
  int N;
  const double *mtab;  // metric table (device)
  int period;          // metric period in entries
  // Arnoldi steps GMRES enqueues per host check of the stop flag; above 1
  // only for operators whose kernels return at once while Ctx::skip is set
  int group = 1;
  virtual void apply(Ctx &c, const T *x, T *y) = 0;
  virtual void precondition(Ctx &c, const T *b, T *x) = 0;
  virtual ~LinearOpsT() = default;
};
using LinearOps = LinearOpsT<double>;
// Arnoldi steps per host check of the GMRES stop flag for operators whose
// kernels honour Ctx::skip: a group costs at most kArnoldiGroup - 1 steps of
// no-op launches after convergence and saves a host round trip per step.
constexpr int kArnoldiGroup = 4;
// Degrees whose Schur action streams the 16 panels C_s X_o of a cell (16 t^2
// doubles) instead of X (m x 4t): fewer bytes from q = 5 (k = 4) on.
__host__ __device__ constexpr bool schur_panels_full(int q) { return q >= 5; }

// Krylov workspace of one vector type: basis (R+1 columns, leading dimension
// ld) and the work vectors of the solver.
template <class T>
struct KrylovBufs {
  T *V, *w, *z, *res, *comb, *corr;
  size_t ld;
  int R;
};

// Bound of a device-side wait of the block ILU(0) factor and sweeps. The
// longest legitimate wait is bounded by one whole factor or sweep (45 ms for
// the factor at 128 x 128 Q4 HDG); 250 ms leaves a wide margin and still ends
// a wait on a row that never comes within a fraction of a second.
constexpr unsigned long long kIluWaitLimitNs = 250ull * 1000 * 1000;

// Block ILU(0) of one form (FixedBlockILU, src/block_ilu.cpp:10-109): fixed
// BSR structure in natural order, numeric blocks and the explicit inverses of
// the factored diagonal blocks. Built on first use (eg_ilu.cu).
struct IluPlan {
  bool built = false;
  int rows = 0, B = 0, nnzb = 0, chunk = 0, chunks = 0, maxl = 0, maxu = 0;
  int *row = nullptr, *col = nullptr, *diag = nullptr, *erow = nullptr;
  int *upd_ptr = nullptr, *upd = nullptr;        // per entry: (target, upper) pairs
  int *fill_ptr = nullptr, *fill_src = nullptr;  // per entry: fill contributions
  double *data = nullptr, *dinv = nullptr, *w = nullptr;
  double *panels16 = nullptr;                    // HDG: 16 panels C_s X_o per cell
  // element/full assembly: the operator's blocks, unfactored (`data` itself
  // while the preconditioner is block Jacobi, a separate array under ILU(0))
  double *asmd = nullptr, *asm_own = nullptr;
  double *work = nullptr;                        // factor slab for large blocks
  unsigned long long *progress = nullptr;        // one counter per CTA of a sweep
  int *abort = nullptr;
  unsigned epoch = 0;
  // bound of every device-side wait of the factor and the sweeps; starve (a
  // test setting) makes every wait on another CTA unreachable
  unsigned long long wait_limit_ns = kIluWaitLimitNs;
  int starve = 0;
  int grid_factor = 0, grid_sweep = 0, sweep_warps = 0, staged = 0, ring = 0, maxrow = 0, maxupd = 0;
  size_t sweep_smem = 0, factor_smem = 0;
  // sweep schedules (forward, backward): per CTA the first position, per
  // position (row, first entry, entry count) and the (owner<<22|slot, column)
  // of each entry's dependency
  int *slot_ptr[2] = {nullptr, nullptr};
  int *meta[2] = {nullptr, nullptr};
  int *deps[2] = {nullptr, nullptr};
};

struct Ctx {
  eg_desc desc{};
  eg_opts opts{};
  int q = 0, p = 0, m = 0, t = 0, n = 0, nf = 0, nu = 0, nl = 0;
  Geo geo{};
  cudaStream_t stream = nullptr;
  std::string err;
  long long bytes = 0;
  std::vector<void *> allocations;

  // tables and metrics
  double *tab = nullptr;
  double *mtab_dg = nullptr, *mtab_hdg = nullptr;
  // body vectors (nu)
  double *u = nullptr, *old = nullptr, *r = nullptr, *du = nullptr, *trial = nullptr,
         *trial_r = nullptr, *er = nullptr, *tmp_body = nullptr;
  // frozen HLL data (nf*q)
  double *fa = nullptr, *fbb = nullptr, *flw = nullptr, *frw = nullptr, *fpen = nullptr;
  // HDG (allocated lazily)
  double *D = nullptr;     // nl
  double *XY = nullptr;    // n*m*(4t+1): per cell [X (m x 4t) | y (m)]
  double *Cb = nullptr;    // n*4q*16 restriction flux blocks C
  double *sf = nullptr;    // n*4q lift scalars B
  double *contrib = nullptr;  // n*4t per-cell face contributions
  // Schur panels C_s X_o of every cell, column-major t x t: the 4 diagonal
  // ones (s = o, the Jacobi blocks) or, where geo.npan == 16
  // (schur_panels_full(q), or element/full assembly), all 16 ([cell][s][o]),
  // which the Schur action then streams instead of X
  double *panels = nullptr;
  double *rhs = nullptr, *lam = nullptr, *tmp_trace = nullptr;  // nl
  double *work_cell = nullptr;  // global LU workspace for large cells
  int work_slots = 0;
  double *work_gj = nullptr;    // k >= 5 condensation: one m x (m + 4t + 1) slab per CTA
  int work_gj_slots = 0;
  // preconditioners (factored in place): DG n blocks m x m, HDG nf blocks t x t;
  // dg_pc_inverse: pc_dg holds explicit inverses (column-major, k <= 2) or a
  // Gauss-Jordan record (k = 3..5, with dg_rec_fac and dg_rec_pivs), else
  // pivoted LU
  double *pc_dg = nullptr, *pc_hdg = nullptr;
  bool dg_pc_inverse = false;
  double *dg_rec_fac = nullptr;
  int *dg_rec_pivs = nullptr;
  // DG partial assembly (launch_dg_refresh): dt w J_x, dt w J_y per cell node
  // and lw J(U_L) + pen I, rw J(U_R) - pen I per face point, component-major
  double *dgc_vol = nullptr, *dgc_face = nullptr;
  double *dgc_h = nullptr;  // face values of the residual and of the cached DG action, 4 per face point
  // --solver dense: the assembled system as a column-major N x N LU with its pivots
  double *dense_a = nullptr;
  int *dense_piv = nullptr;
  int dense_n = 0;
  int *piv_dg = nullptr, *piv_hdg = nullptr;
  // Krylov workspace (size N = max(nu, nl) so both forms share it)
  int kN = 0, kR = 0;
  double *V = nullptr;
  double *kw = nullptr, *kz = nullptr, *kres = nullptr, *kcomb = nullptr, *kcorr = nullptr,
         *kx = nullptr;
  GmresCtl *ctl = nullptr;
  GmresCtl *hctl = nullptr;  // pinned mirror
  // set while GMRES enqueues a group of Arnoldi steps: the operator kernels
  // of those steps return at once when *skip (the device stop flag) is set
  const int *skip = nullptr;
  double *partials = nullptr;  // kRedBlocks * (kMaxRestart+1)
  unsigned *counter = nullptr;
  // error word (derr[0]) and admissibility flag (derr[1])
  int *derr = nullptr;
  double *dscal = nullptr;
  double *field_partial = nullptr;  // per-cell partials of the diagnostics (4n) and their sum (4)
  double *hscal = nullptr;  // pinned mirror of dscal
  int *herr = nullptr;      // pinned
  // events for per-update device timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_residual_s = 0.;
  bool update_timer_open = false;

  IluPlan ilu[2];  // per form (EG_FORM_DG, EG_FORM_HDG)
  unsigned long long ilu_wait_limit_ns = kIluWaitLimitNs;  // eg_set_ilu_wait
  int ilu_starve = 0;
  double *step_bufs = nullptr;  // time loop: step state, stage base, 4 slopes (6 nu), reused
  // mixed precision: FP32 copies of X, of the Schur block-Jacobi inverses and
  // of D, and the FP32 Krylov workspace of the inner Schur solve
  // mixed precision: Xf is the FP32 copy of X, or of the 16 Schur panels per
  // cell where geo.npan == 16
  float *Xf = nullptr, *pcf = nullptr, *Df = nullptr, *contribf = nullptr;
  float *kfV = nullptr, *kfw = nullptr, *kfz = nullptr, *kfres = nullptr, *kfcomb = nullptr,
        *kfcorr = nullptr, *kfx = nullptr, *kfrhs = nullptr;

  bool residual_ready = false;
  bool condensed = false;
  // set when an aborted sweep's bulk copy did not land within its bound: the
  // context's device memory can no longer be trusted; only eg_destroy works
  bool broken = false;
  Profiler prof;
  long long launches = 0;

  void *alloc(size_t bytes);
  template <class T>
  T *alloc_n(size_t n) {
    return static_cast<T *>(alloc(n * sizeof(T)));
  }
  void ensure_hdg();
  void ensure_krylov();
  void ensure_pc_dg();
  void ensure_pc_hdg();
  void sync();
  void check_device_error();
  void prof_resolve();
};

// ---- launchers (eg_cell.cu) ----
void launch_freeze(Ctx &c, const double *u, bool check_admissible);
void launch_admissible(Ctx &c, const double *u);  // writes dscal[DS_ADMISSIBLE]
void launch_residual(Ctx &c, const double *u, const double *old, double *r);
void launch_dg_apply(Ctx &c, const double *u, const double *x, double *y);  // Jacobians recomputed
// PartialDGOperator::Refresh at state u, then the cached action (Mult)
void launch_dg_refresh(Ctx &c, const double *u);
void launch_dg_apply_cached(Ctx &c, const double *x, double *y);
// ---- dense direct solve of the full assembly (eg_dense.cu) ----
constexpr int kDenseMaxUnknowns = 5000;
void dense_factor(Ctx &c, int form);  // LU of the assembled blocks of c.ilu[form]
void dense_solve(Ctx &c, const double *b, double *x);
void launch_dg_jacobi(Ctx &c, const double *u, bool factor);
void launch_block_apply(Ctx &c, const double *blocks, const int *piv, int nblocks, int bs,
                        const double *b, double *x);
// DG block-Jacobi apply x = J_KK^{-1} b with whichever factors the last
// launch_dg_jacobi(factor = true) formed (explicit inverses or pivoted LU).
void launch_dg_jacobi_apply(Ctx &c, const double *b, double *x);
// ---- explicit DG block-Jacobi inverses (eg_dginv.cu) ----
bool dg_inverse_supported(int q);
// k <= 2: pc_dg holds the column-major J_KK^{-1}; k = 3..5: the Gauss-Jordan
// record (pc_dg: reduced block, dg_rec_fac: panel T^{-1}, dg_rec_pivs: panel
// pivot rows, piv_dg: unknown order of the result rows)
bool dg_pc_is_record(const Ctx &c);
void launch_dg_inverse(Ctx &c, const double *u);
void launch_dg_inverse_apply(Ctx &c, const double *b, double *x);
// the explicit inverses a record applies, column-major (n m^2 doubles, host)
void download_dg_record_inverse(Ctx &c, double *dst);
// ---- launchers (eg_hdg.cu) ----
void launch_condense(Ctx &c, const double *u, const double *r);
void launch_schur_apply(Ctx &c, const double *v, double *y);
void launch_recover(Ctx &c, const double *lam, double *du);
void launch_recovered_residual(Ctx &c, const double *eq, double *er);
void launch_schur_jacobi(Ctx &c, bool factor);
// x = Inv b for explicit block inverses (Schur block Jacobi apply).
void launch_block_inverse_apply(Ctx &c, const double *inv, int nblocks, int bs, const double *b, double *x);
// in-place transpose of every bs x bs block of `a`
void launch_transpose_blocks(Ctx &c, double *a, int nblocks, int bs);
// ---- eg_api.cu ----
// Sets the context's description (geometry, tables, metrics) for its size.
void upload_desc(Ctx &c, const eg_desc &d);
// ---- initial projection and diagnostics (eg_field.cu) ----
// u <- L2 projection of the exact wave at t = 0 (Problem::Initial).
void field_initial(Ctx &c, double *u);
// L2 errors against the exact wave at `time` (Problem::Errors), conserved
// integrals (Problem::Integral) and L2 norms of u - v (Problem::Differences)
// of device body vectors; each synchronises the stream and returns on the host.
void field_errors(Ctx &c, const double *u, double time, double out[4]);
void field_integral(Ctx &c, const double *u, double out[4]);
void field_differences(Ctx &c, const double *u, const double *v, double out[4]);
// ---- block ILU(0) (eg_ilu.cu) ----
// Fill (and with factor set, factor) the ILU of `form` at the current state /
// condensation; x = ILU^{-1} b.
void ilu_refresh(Ctx &c, int form, bool factor);
void launch_ilu_apply(Ctx &c, int form, const double *b, double *x);
// ---- element/full assembly (eg_ilu.cu) ----
// Fill the assembled block-sparse operator of `form` (the ILU(0) block
// structure, unfactored) at the current state / condensation; y = A x.
void assemble_blocks(Ctx &c, int form);
void launch_assembled_apply(Ctx &c, int form, const double *x, double *y);
// ---- mixed precision (eg_mixed.cu) ----
// FP32 copies of the condensed responses and of the factored Schur
// block-Jacobi inverses (after eg_condense and the FP64 factor).
void mixed_prepare(Ctx &c);
// S x = rhs by FP64 iterative refinement around an FP32 inner GMRES; leaves
// rhs - S x in c.kres and returns its weighted norm. *count = inner iterations.
double schur_refine_mixed(Ctx &c, const double *rhs, double *x, bool zero_guess, double tol, int limit,
                          double rhs_norm, int *count);
// ---- launchers (eg_krylov.cu) ----
// Weighted squared norm sum(metric * x * x) into dscal[slot] (device).
void launch_wnorm2(Ctx &c, const double *x, int N, const double *mtab, int period, int slot);
double wnorm(Ctx &c, const double *x, int N, const double *mtab, int period);
void launch_axpby(Ctx &c, int N, double a, const double *x, double b, const double *y, double *out);
void launch_copy(Ctx &c, int N, const double *x, double *out);
void launch_fill(Ctx &c, int N, double v, double *out);
double cell_norm(Ctx &c, const double *x);
// Weighted restarted GMRES (src/linear.cpp:76-157). Returns the true residual
// norm; sets *count. Throws Failure on breakdown / limit / non-finite.
// known_rhs_norm >= 0 is the caller's weighted norm of rhs (saves a reduction
// and a host round trip).
double gmres(Ctx &c, LinearOps &ops, const double *rhs, double *x, double tol, int limit,
             bool zero_guess, int *count, double *rhs_norm_out, double known_rhs_norm = -1.);
// The same iteration on FP32 vectors from a zero guess; returns the residual
// norm reached without requiring convergence (inner solve of mixed precision).
double gmres_f32(Ctx &c, LinearOpsT<float> &ops, const KrylovBufs<float> &kb, const float *rhs, float *x,
                 double tol, int limit, int *count);
// ---- eg_api.cu ----
// One accepted damped Newton update (src/stepper.cpp:129-228).
void newton_update(Ctx &c, double residual_norm, double old_norm, eg_update_stats *st);

}  // namespace eg
