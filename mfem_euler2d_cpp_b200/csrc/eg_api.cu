// C-ABI implementation: context lifetime, state transfer, operator entry
// points and the device-resident Newton update (src/stepper.cpp:116-228).
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "eg_internal.h"
#include "eg_setup.h"

struct eg_ctx {
  eg::Ctx c;
};

namespace eg {

void fail(int status, const std::string &msg) { throw Failure{status, msg}; }

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) fail(EG_ERR_OUT_OF_MEMORY, std::string(what) + ": out of memory");
  fail(EG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static const char *kMessages[EG_ERR_COUNT] = {
    "ok",
    "invalid argument",
    "CUDA error",
    "Nonpositive old face state; refine mesh",
    "Invalid Roe sound speed",
    "Degenerate HLL speeds",
    "Old state is inadmissible; refine mesh",
    "Singular streaming HDG cell factor",
    "Singular block Jacobi factor",
    "Singular BSR ILU diagonal",
    "GMRES Arnoldi breakdown",
    "Nonfinite GMRES residual",
    "GMRES iteration limit reached",
    "True inverse-mass weighted linear residual too large",
    "Recovered DG residual criterion failed after Schur refinement",
    "DG Newton linear residual too large",
    "Newton line search failed",
    "device out of memory",
    "Step leaves the smooth simple-wave interval T < 4/((gamma+1)*pi)",
    "Newton failed to converge",
    "SSP-DIRK3 step produced an inadmissible state",
    "Initial projection not positive; refine mesh",
    "Independent recovered DG equation check failed",
    "DG/HDG one-update equivalence failed",
    "device wait limit reached",
    "context lost: a bulk copy of an aborted sweep did not finish; destroy the context",
};

void *Ctx::alloc(size_t nbytes) {
  void *p = nullptr;
  const cudaError_t e = cudaMalloc(&p, std::max<size_t>(nbytes, 16));
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(EG_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(nbytes) + " bytes failed");
  }
  allocations.push_back(p);
  bytes += (long long)nbytes;
  return p;
}

void Ctx::sync() { EG_CUDA(cudaStreamSynchronize(stream)); }

static cudaEvent_t take_event(Ctx &c) {
  if (!c.prof.pool.empty()) {
    cudaEvent_t e = c.prof.pool.back();
    c.prof.pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  EG_CUDA(cudaEventCreate(&e));
  return e;
}

ProfScope::ProfScope(Ctx &ctx, int kernel_class, long long nlaunch)
    : c(ctx), id(kernel_class), launches(nlaunch) {
  c.launches += nlaunch;
  if (c.prof.on) {
    a = take_event(c);
    b = take_event(c);
    cudaEventRecord(a, c.stream);
  }
}
ProfScope::~ProfScope() {
  if (a) {
    cudaEventRecord(b, c.stream);
    c.prof.pending.push_back({id, launches, a, b});
    if (c.prof.pending.size() > 4096) {
      cudaStreamSynchronize(c.stream);
      c.prof_resolve();
    }
  }
}

void Ctx::prof_resolve() {
  for (auto &r : prof.pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      prof.ms[r.id] += ms;
      prof.count[r.id] += r.launches;
    }
    prof.pool.push_back(r.a);
    prof.pool.push_back(r.b);
  }
  prof.pending.clear();
}

void Ctx::check_device_error() {
  EG_CUDA(cudaMemcpyAsync(herr, derr, sizeof(int), cudaMemcpyDeviceToHost, stream));
  EG_CUDA(cudaMemcpyAsync(herr + 2, derr + 2, sizeof(int), cudaMemcpyDeviceToHost, stream));
  sync();
  if (herr[2]) {
    broken = true;
    fail(EG_ERR_CONTEXT_LOST, kMessages[EG_ERR_CONTEXT_LOST]);
  }
  const int code = *herr;
  if (code != 0) {
    EG_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), stream));
    sync();
    fail(code, code < EG_ERR_COUNT ? kMessages[code] : "device error");
  }
}

void Ctx::ensure_hdg() {
  if (XY) return;
  XY = alloc_n<double>((size_t)n * m * (4 * t + 1));
  Cb = alloc_n<double>((size_t)n * 4 * q * 16);
  sf = alloc_n<double>((size_t)n * 4 * q);
  contrib = alloc_n<double>((size_t)n * 4 * t);
  panels = alloc_n<double>((size_t)n * geo.npan * t * t);
  rhs = alloc_n<double>(nl);
  lam = alloc_n<double>(nl);
  tmp_trace = alloc_n<double>(nl);
  EG_CUDA(cudaMemsetAsync(lam, 0, sizeof(double) * nl, stream));
}

void Ctx::ensure_krylov() {
  if (V) return;
  kN = std::max(nu, nl);
  kR = opts.restart;
  V = alloc_n<double>((size_t)kN * (kR + 1));
  kw = alloc_n<double>(kN);
  kz = alloc_n<double>(kN);
  kres = alloc_n<double>(kN);
  kcomb = alloc_n<double>(kN);
  kcorr = alloc_n<double>(kN);
}

void Ctx::ensure_pc_dg() {
  if (pc_dg) return;
  pc_dg = alloc_n<double>((size_t)n * m * m);
  piv_dg = alloc_n<int>((size_t)n * m);
}
void Ctx::ensure_pc_hdg() {
  if (pc_hdg) return;
  pc_hdg = alloc_n<double>((size_t)nf * t * t);
  piv_hdg = alloc_n<int>((size_t)nf * t);
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------ linear ops
struct DgOps : LinearOps {
  explicit DgOps(Ctx &c) {
    N = c.nu;
    mtab = c.mtab_dg;
    period = c.m;
  }
  // partial assembly: the Jacobians cached by the refresh at the start of
  // the solve; element/full: the assembled cell and face-coupling blocks
  void apply(Ctx &c, const double *x, double *y) override {
    if (c.opts.assembly == EG_ASSEMBLY_PARTIAL)
      launch_dg_apply_cached(c, x, y);
    else
      launch_assembled_apply(c, EG_FORM_DG, x, y);
  }
  void precondition(Ctx &c, const double *b, double *x) override {
    if (c.opts.precond == EG_PC_BLOCK_ILU0)
      launch_ilu_apply(c, EG_FORM_DG, b, x);
    else
      launch_dg_jacobi_apply(c, b, x);
  }
};
struct HdgOps : LinearOps {
  explicit HdgOps(Ctx &c) {
    N = c.nl;
    mtab = c.mtab_hdg;
    period = 2 * c.t;
    // the block-Jacobi and Schur kernels honour Ctx::skip; the ILU sweeps do not
    group = c.opts.precond == EG_PC_BLOCK_ILU0 ? 1 : kArnoldiGroup;
  }
  // partial/element: the per-cell Schur action; full: the assembled matrix
  void apply(Ctx &c, const double *x, double *y) override {
    if (c.opts.assembly == EG_ASSEMBLY_FULL)
      launch_assembled_apply(c, EG_FORM_HDG, x, y);
    else
      launch_schur_apply(c, x, y);
  }
  void precondition(Ctx &c, const double *b, double *x) override {
    if (c.opts.precond == EG_PC_BLOCK_ILU0)
      launch_ilu_apply(c, EG_FORM_HDG, b, x);
    else
      launch_block_inverse_apply(c, c.pc_hdg, c.nf, c.t, b, x);
  }
};

static void pc_factor(Ctx &c, int form, bool factor) {
  if (c.opts.precond == EG_PC_BLOCK_ILU0) {
    // FillBlocks + FixedBlockILU::Factor (src/linear.cpp:191, 196-197)
    ilu_refresh(c, form, factor);
  } else if (form == EG_FORM_DG) {
    launch_dg_jacobi(c, c.u, factor);
  } else {
    if (!c.condensed) fail(EG_ERR_INVALID, "Schur preconditioner requires a condensation");
    launch_schur_jacobi(c, factor);
  }
  c.check_device_error();
}

// LinearSolver::Solve (src/linear.cpp:167-249). x is the initial guess when
// refresh is false; eq receives op*x - rhs.
struct LinearOut {
  int count = 0;
  double residual = 0., rhs_norm = 0., assembly = 0., setup = 0., solve = 0.;
};
static void linear_solve(Ctx &c, int form, const double *rhs, double *x, double *eq, bool refresh,
                         double tol, LinearOut &out) {
  DgOps dg(c);
  HdgOps hdg(c);
  LinearOps &ops = form == EG_FORM_DG ? static_cast<LinearOps &>(dg) : static_cast<LinearOps &>(hdg);
  out = LinearOut();
  // the residual and work vectors below live in the Krylov workspace, which
  // the dense solve needs as well
  c.ensure_krylov();
  const double rhs_norm = wnorm(c, rhs, ops.N, ops.mtab, ops.period);
  out.rhs_norm = rhs_norm;
  if (rhs_norm == 0.) {
    launch_fill(c, ops.N, 0., x);
    if (eq) launch_fill(c, ops.N, 0., eq);
    return;
  }
  // assembled operator: ElementOperator::Assemble for full assembly and the
  // element-assembled DG Jacobian (src/linear.cpp:186-190, stepper.cpp:139-140);
  // the element-assembled Schur entries come with the condensation
  const bool assembled = form == EG_FORM_DG ? c.opts.assembly != EG_ASSEMBLY_PARTIAL
                                            : c.opts.assembly == EG_ASSEMBLY_FULL;
  double t0 = now_s();
  // DG partial assembly: PartialDGOperator::Refresh at the Newton state
  // (src/stepper.cpp:139), kept for the whole solve like the reference's
  if (form == EG_FORM_DG && c.opts.assembly == EG_ASSEMBLY_PARTIAL && (refresh || !c.dgc_vol))
    launch_dg_refresh(c, c.u);
  if (refresh && assembled) assemble_blocks(c, form);
  out.assembly = now_s() - t0;
  t0 = now_s();
  const bool dense = c.opts.solver == EG_SOLVER_DENSE;
  if (refresh) {
    if (dense)
      dense_factor(c, form);  // src/linear.cpp:204-206 (no preconditioner)
    else
      pc_factor(c, form, true);
  }
  out.setup = now_s() - t0;
  t0 = now_s();
  int count = 0;
  // mixed precision: FP32 inner solve of the condensed system in FP64
  // refinement (block Jacobi only; DG and block ILU(0) stay FP64)
  const bool mixed = c.opts.precision == EG_PRECISION_MIXED && form == EG_FORM_HDG &&
                     c.opts.precond == EG_PC_BLOCK_JACOBI;
  double res = 0.;
  try {
    if (dense) {
      dense_solve(c, rhs, x);  // src/linear.cpp:224-225; the residual follows below
    } else if (mixed) {
      if (refresh) mixed_prepare(c);
      res = schur_refine_mixed(c, rhs, x, refresh, tol, c.opts.max_krylov, rhs_norm, &count);
    } else {
      res = gmres(c, ops, rhs, x, tol, c.opts.max_krylov, refresh, &count, nullptr, rhs_norm);
    }
  } catch (const Failure &) {
    c.check_device_error();  // a preconditioner failure on the device explains the breakdown
    throw;
  }
  c.check_device_error();
  out.solve = now_s() - t0;
  out.count = count;
  if (c.opts.assembly == EG_ASSEMBLY_FULL) {
    // GMRES ran on the assembled matrix: the residual comes from the
    // element operator's own action (src/linear.cpp:242-246)
    double *dst = eq ? eq : c.kres;
    if (form == EG_FORM_DG)
      launch_dg_apply(c, c.u, x, c.kw);
    else
      launch_schur_apply(c, x, c.kw);
    launch_axpby(c, ops.N, 1., c.kw, -1., rhs, dst);
    res = wnorm(c, dst, ops.N, ops.mtab, ops.period);
  } else if (eq) {
    launch_axpby(c, ops.N, -1., c.kres, 0., c.kres, eq);
  }
  out.residual = res / rhs_norm;
  if (!(std::isfinite(out.residual) && out.residual <= std::max(10 * tol, 1e-12)))
    fail(EG_ERR_LINEAR_RESIDUAL, "True inverse-mass weighted linear residual too large");
}

static void open_update_timer(Ctx &c) {
  EG_CUDA(cudaEventRecord(c.ev0, c.stream));
  c.update_timer_open = true;
}

void newton_update(Ctx &c, double residual_norm, double old_norm, eg_update_stats *st) {
  eg_update_stats s{};
  const double t_begin = now_s();
  if (!c.update_timer_open) open_update_timer(c);
  const int form = c.opts.form;
  const double eps = std::numeric_limits<double>::epsilon();
  const double allowance = 128 * eps * (cell_norm(c, c.u) + old_norm + residual_norm);
  const double target = std::max(10 * c.opts.linear_tol * residual_norm, allowance);
  double er_norm = 0.;
  LinearOut lr;
  int total_count = 0;
  if (form == EG_FORM_DG) {
    // Jacobians are evaluated from the Newton state inside every action.
    launch_axpby(c, c.nu, -1., c.r, 0., c.r, c.tmp_body);
    linear_solve(c, EG_FORM_DG, c.tmp_body, c.du, c.er, true, c.opts.linear_tol, lr);
    total_count = lr.count;
    s.assembly_s = lr.assembly;
    s.setup_s = lr.setup;
    s.solve_s = lr.solve;
    const double v0 = now_s();
    er_norm = cell_norm(c, c.er);
    s.validation_s = now_s() - v0;
  } else {
    const double c0 = now_s();
    launch_condense(c, c.u, c.r);
    c.check_device_error();
    s.condensation_s = now_s() - c0;
    double tol = c.opts.linear_tol;
    bool valid = false;
    for (int attempt = 0; attempt < 4; ++attempt) {
      LinearOut a;
      linear_solve(c, EG_FORM_HDG, c.rhs, c.lam, c.tmp_trace, attempt == 0, tol, a);
      total_count += a.count;
      s.assembly_s += a.assembly;
      s.setup_s += a.setup;
      s.solve_s += a.solve;
      lr.residual = a.residual;
      const double r0 = now_s();
      launch_recover(c, c.lam, c.du);
      c.sync();
      s.recovery_s += now_s() - r0;
      const double v0 = now_s();
      launch_recovered_residual(c, c.tmp_trace, c.er);
      er_norm = cell_norm(c, c.er);
      s.validation_s += now_s() - v0;
      s.attempts = attempt + 1;
      valid = er_norm <= target;
      if (valid) break;
      tol *= .01;
    }
    if (!valid) fail(EG_ERR_RECOVERED, "Recovered DG residual criterion failed after Schur refinement");
  }
  s.krylov_iterations = total_count;
  s.linear_relative_residual = form == EG_FORM_DG ? lr.residual : lr.residual;
  s.dg_linear_relative_residual = residual_norm > 0 ? er_norm / residual_norm : 0.;
  if (!(er_norm <= target)) fail(EG_ERR_DG_LINEAR, "DG Newton linear residual too large");
  // --check-update: independent DG equation and solve of the recovered HDG
  // increment (src/stepper.cpp:184-201); excluded from the update time.
  double diagnostic_s = 0.;
  s.update_check = -1.;
  if (c.opts.check_update && form == EG_FORM_HDG) {
    const double d0 = now_s();
    launch_dg_apply(c, c.u, c.du, c.tmp_body);
    launch_axpby(c, c.nu, 1., c.tmp_body, 1., c.r, c.tmp_body);
    if (!(cell_norm(c, c.tmp_body) <= std::max(4 * target, 1e-12)))
      fail(EG_ERR_UPDATE_EQUATION, "Independent recovered DG equation check failed");
    launch_axpby(c, c.nu, -1., c.r, 0., c.r, c.tmp_body);
    LinearOut ref;
    linear_solve(c, EG_FORM_DG, c.tmp_body, c.er, nullptr, true, c.opts.linear_tol, ref);
    launch_axpby(c, c.nu, 1., c.du, -1., c.er, c.tmp_body);
    const double diff = cell_norm(c, c.tmp_body), refn = cell_norm(c, c.er);
    s.update_check = diff / std::max(refn, 1e-30);
    if (!(diff <= std::max(1e-8 * refn, 4 * allowance)))
      fail(EG_ERR_UPDATE_EQUIVALENCE, "DG/HDG one-update equivalence failed");
    diagnostic_s = now_s() - d0;
  }
  // damped line search (src/stepper.cpp:202-222)
  const double ls0 = now_s();
  double damping = 1.;
  bool accept = false;
  for (int back = 0; back < 30; ++back) {
    launch_axpby(c, c.nu, 1., c.u, damping, c.du, c.trial);
    launch_admissible(c, c.trial);
    EG_CUDA(cudaMemcpyAsync(c.herr + 1, c.derr + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (c.herr[1]) {
      launch_residual(c, c.trial, c.old, c.trial_r);
      if (cell_norm(c, c.trial_r) <= (1 - 1e-4 * damping) * residual_norm + allowance) {
        accept = true;
        break;
      }
    }
    damping *= .5;
  }
  if (!accept) fail(EG_ERR_LINE_SEARCH, "Newton line search failed");
  std::swap(c.u, c.trial);
  std::swap(c.r, c.trial_r);
  c.residual_ready = true;
  s.line_search_s = now_s() - ls0;
  s.damping = damping;
  s.residual_norm = residual_norm;
  EG_CUDA(cudaEventRecord(c.ev1, c.stream));
  c.sync();
  float ms = 0.f;
  EG_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  c.update_timer_open = false;
  s.device_ms = ms;
  s.residual_s = c.last_residual_s;
  s.iteration_s = c.last_residual_s + (now_s() - t_begin) - diagnostic_s;
  if (st) *st = s;
}

// Geometry and tables of the description (tab: [tdx][tdy][fb][w][inv_mass]
// [mass][ew]; dual-norm metric tables), uploaded in stream order.
void upload_desc(Ctx &c, const eg_desc &d) {
  c.desc = d;
  c.geo = Geo{d.nx, d.ny, c.n, c.nf, d.hx, d.hy, d.area, c.geo.dt, d.gamma, d.gamma - 1., d.safety,
              schur_panels_full(c.q) || c.opts.assembly != EG_ASSEMBLY_PARTIAL ? 16 : 4};
  const int q = c.q, p = c.p;
  std::vector<double> tab(tab_size(q));
  for (int i = 0; i < p; ++i) {
    tab[i] = d.tensor_dx[i];
    tab[p + i] = d.tensor_dy[i];
    tab[6 * p + i] = d.w[i];
    tab[7 * p + i] = d.inv_mass[i];
    tab[8 * p + i] = d.mass[i];
  }
  for (int i = 0; i < 4 * p; ++i) tab[2 * p + i] = d.face_basis[i];
  for (int j = 0; j < q; ++j) tab[9 * p + j] = d.ew[j];
  std::vector<double> mdg(p), mhdg(2 * q);
  for (int i = 0; i < p; ++i) mdg[i] = d.area * d.mass[i];
  for (int j = 0; j < q; ++j) {
    mhdg[j] = d.hy / d.ew[j];
    mhdg[q + j] = d.hx / d.ew[j];
  }
  EG_CUDA(cudaMemcpyAsync(c.tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c.stream));
  EG_CUDA(cudaMemcpyAsync(c.mtab_dg, mdg.data(), sizeof(double) * p, cudaMemcpyHostToDevice, c.stream));
  EG_CUDA(cudaMemcpyAsync(c.mtab_hdg, mhdg.data(), sizeof(double) * 2 * q, cudaMemcpyHostToDevice, c.stream));
  c.sync();  // the host tables are local
  c.residual_ready = false;
  c.condensed = false;
}

static double *slot_ptr(Ctx &c, int slot, size_t &count) {
  switch (slot) {
    case EG_SLOT_U: count = c.nu; return c.u;
    case EG_SLOT_OLD: count = c.nu; return c.old;
    case EG_SLOT_R: count = c.nu; return c.r;
    case EG_SLOT_DU: count = c.nu; return c.du;
    case EG_SLOT_RHS: c.ensure_hdg(); count = c.nl; return c.rhs;
    case EG_SLOT_LAMBDA: c.ensure_hdg(); count = c.nl; return c.lam;
    case EG_SLOT_D: count = c.nl; return c.D;
    case EG_SLOT_HLL_A: count = (size_t)c.nf * c.q; return c.fa;
    case EG_SLOT_HLL_B: count = (size_t)c.nf * c.q; return c.fbb;
    default: fail(EG_ERR_INVALID, "invalid slot");
  }
}

static void upload_vec(Ctx &c, double *dst, const double *src, size_t count) {
  if (!src) fail(EG_ERR_INVALID, "null vector");
  EG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDefault, c.stream));
}
static void download_vec(Ctx &c, double *dst, const double *src, size_t count) {
  if (!dst) fail(EG_ERR_INVALID, "null vector");
  EG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDefault, c.stream));
  c.sync();
}

}  // namespace eg

using eg::Ctx;
using eg::Failure;

// Message of the last failed eg_create on this thread (no context exists then).
static thread_local std::string g_create_error;

template <class F>
static int guard(eg_ctx *ctx, F &&f) {
  if (ctx && ctx->c.broken) {
    ctx->c.err = eg::kMessages[EG_ERR_CONTEXT_LOST];
    return EG_ERR_CONTEXT_LOST;
  }
  try {
    f();
    return EG_OK;
  } catch (const Failure &e) {
    if (ctx) ctx->c.err = e.msg;
    return e.status;
  } catch (const std::exception &e) {
    if (ctx) ctx->c.err = e.what();
    return EG_ERR_INVALID;
  }
}

extern "C" {

const char *eg_status_string(int status) {
  if (status < 0 || status >= EG_ERR_COUNT) return "unknown status";
  return eg::kMessages[status];
}

const char *eg_last_error(const eg_ctx *ctx) { return ctx ? ctx->c.err.c_str() : g_create_error.c_str(); }

int eg_desc_simple_wave(eg_desc *d, int nx, int ny, int k, double alpha_deg, double gamma,
                        double safety) {
  if (!d) return EG_ERR_INVALID;
  try {
    eg::host::fill_desc(*d, nx, ny, k, alpha_deg, gamma, safety);
  } catch (const std::exception &) {
    return EG_ERR_INVALID;
  }
  return EG_OK;
}

int eg_set_device(int device) {
  const cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    g_create_error = cudaGetErrorString(e);
    return EG_ERR_CUDA;
  }
  return EG_OK;
}

void eg_opts_default(eg_opts *o) {
  o->form = EG_FORM_HDG;
  o->precond = EG_PC_BLOCK_JACOBI;
  o->assembly = EG_ASSEMBLY_PARTIAL;
  o->precision = EG_PRECISION_FP64;
  o->restart = 20;
  o->max_krylov = 1500;
  o->linear_tol = 1e-12;
  o->check_update = 0;
  o->solver = EG_SOLVER_GMRES;
}

static void validate_opts(const eg_opts &o) {
  if (o.form != EG_FORM_DG && o.form != EG_FORM_HDG) eg::fail(EG_ERR_INVALID, "Invalid form");
  if (o.precond != EG_PC_BLOCK_JACOBI && o.precond != EG_PC_BLOCK_ILU0)
    eg::fail(EG_ERR_INVALID, "Invalid preconditioner");
  if (o.restart <= 0 || o.max_krylov <= 0) eg::fail(EG_ERR_INVALID, "Iteration limits must be positive");
  if (o.restart > eg::kMaxRestart) eg::fail(EG_ERR_INVALID, "restart above the supported maximum of 64");
  if (!(o.linear_tol > 0)) eg::fail(EG_ERR_INVALID, "linear tolerance must be positive");
  if (o.precision != EG_PRECISION_FP64 && o.precision != EG_PRECISION_MIXED)
    eg::fail(EG_ERR_INVALID, "Invalid precision");
  if (o.assembly != EG_ASSEMBLY_PARTIAL && o.assembly != EG_ASSEMBLY_ELEMENT && o.assembly != EG_ASSEMBLY_FULL)
    eg::fail(EG_ERR_INVALID, "Invalid assembly");
  if (o.precision == EG_PRECISION_MIXED && o.assembly == EG_ASSEMBLY_FULL)
    eg::fail(EG_ERR_INVALID, "mixed precision requires partial or element assembly");
  if (o.solver != EG_SOLVER_GMRES && o.solver != EG_SOLVER_DENSE) eg::fail(EG_ERR_INVALID, "Invalid solver");
  if (o.solver == EG_SOLVER_DENSE && o.assembly != EG_ASSEMBLY_FULL)
    eg::fail(EG_ERR_INVALID, "Direct LU requires --assembly full");
}
// LinearSolver workspace (src/linear.cpp:46-47): the dense solve's size limit
static void validate_dense_size(const Ctx &c) {
  if (c.opts.solver != EG_SOLVER_DENSE) return;
  const long long n = c.opts.form == EG_FORM_DG ? (long long)c.nu : (long long)c.nl;
  if (n > eg::kDenseMaxUnknowns) eg::fail(EG_ERR_INVALID, "Dense direct solve limited to 5000 unknowns");
}

int eg_create(const eg_desc *d, const eg_opts *o, eg_ctx **out) {
  if (!d || !o || !out) return EG_ERR_INVALID;
  *out = nullptr;
  auto *ctx = new eg_ctx();
  Ctx &c = ctx->c;
  const int rc = guard(ctx, [&] {
    if (d->k < 0 || d->k > 8 || d->nx < 2 || d->ny < 2)
      eg::fail(EG_ERR_INVALID, "Invalid mesh or degree");
    validate_opts(*o);
    c.desc = *d;
    c.opts = *o;
    c.q = d->k + 1;
    c.p = c.q * c.q;
    c.m = 4 * c.p;
    c.t = 4 * c.q;
    c.n = d->nx * d->ny;
    c.nf = 2 * c.n;
    const long double nu = 4.L * c.n * c.p, nl = 8.L * c.n * c.q;
    if (nu > std::numeric_limits<int>::max() || nl > std::numeric_limits<int>::max())
      eg::fail(EG_ERR_INVALID, "Mesh/degree exceeds int DOF capacity");
    c.nu = c.n * c.m;
    c.nl = c.nf * c.t;
    validate_dense_size(c);
    for (int i = 0; i < c.p; ++i)
      if (d->tensor_node[i] != i)
        eg::fail(EG_ERR_INVALID, "native node order must be lexicographic (x fastest)");
    EG_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    EG_CUDA(cudaEventCreate(&c.ev0));
    EG_CUDA(cudaEventCreate(&c.ev1));
    const int q = c.q;
    c.tab = c.alloc_n<double>(eg::tab_size(q));
    c.mtab_dg = c.alloc_n<double>(c.p);
    c.mtab_hdg = c.alloc_n<double>(2 * q);
    eg::upload_desc(c, *d);
    for (double **v : {&c.u, &c.old, &c.r, &c.du, &c.trial, &c.trial_r, &c.er, &c.tmp_body}) {
      *v = c.alloc_n<double>(c.nu);
      EG_CUDA(cudaMemsetAsync(*v, 0, sizeof(double) * c.nu, c.stream));
    }
    for (double **v : {&c.fa, &c.fbb, &c.flw, &c.frw, &c.fpen}) {
      *v = c.alloc_n<double>((size_t)c.nf * q);
      EG_CUDA(cudaMemsetAsync(*v, 0, sizeof(double) * c.nf * q, c.stream));
    }
    c.D = c.alloc_n<double>(c.nl);
    EG_CUDA(cudaMemsetAsync(c.D, 0, sizeof(double) * c.nl, c.stream));
    c.derr = c.alloc_n<int>(4);
    EG_CUDA(cudaMemsetAsync(c.derr, 0, 4 * sizeof(int), c.stream));
    c.dscal = c.alloc_n<double>(eg::DS_COUNT);
    EG_CUDA(cudaMemsetAsync(c.dscal, 0, eg::DS_COUNT * sizeof(double), c.stream));
    c.counter = c.alloc_n<unsigned>(1);
    EG_CUDA(cudaMemsetAsync(c.counter, 0, sizeof(unsigned), c.stream));
    c.partials = c.alloc_n<double>((size_t)eg::kRedBlocks * (eg::kMaxRestart + 1));
    c.ctl = c.alloc_n<eg::GmresCtl>(1);
    EG_CUDA(cudaMallocHost(&c.hctl, sizeof(eg::GmresCtl)));
    EG_CUDA(cudaMallocHost(&c.hscal, sizeof(double) * eg::DS_COUNT));
    EG_CUDA(cudaMallocHost(&c.herr, sizeof(int) * 4));
    if (o->form == EG_FORM_HDG) c.ensure_hdg();
    c.sync();
  });
  if (rc != EG_OK) {
    g_create_error = c.err;
    eg_destroy(ctx);
    return rc;
  }
  g_create_error.clear();
  *out = ctx;
  return EG_OK;
}

void eg_destroy(eg_ctx *ctx) {
  if (!ctx) return;
  Ctx &c = ctx->c;
  if (c.stream) cudaStreamSynchronize(c.stream);
  for (auto &r : c.prof.pending) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : c.prof.pool) cudaEventDestroy(e);
  for (void *p : c.allocations) cudaFree(p);
  if (c.hctl) cudaFreeHost(c.hctl);
  if (c.hscal) cudaFreeHost(c.hscal);
  if (c.herr) cudaFreeHost(c.herr);
  if (c.ev0) cudaEventDestroy(c.ev0);
  if (c.ev1) cudaEventDestroy(c.ev1);
  if (c.stream) cudaStreamDestroy(c.stream);
  delete ctx;
}

void *eg_stream(eg_ctx *ctx) { return ctx ? (void *)ctx->c.stream : nullptr; }

int eg_set_opts(eg_ctx *ctx, const eg_opts *o) {
  if (!ctx || !o) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    validate_opts(*o);
    if (o->restart > ctx->c.kR && ctx->c.V) eg::fail(EG_ERR_INVALID, "restart cannot grow after first solve");
    if (o->assembly != ctx->c.opts.assembly)
      eg::fail(EG_ERR_INVALID, "assembly is fixed when the context is created");
    ctx->c.opts = *o;
    validate_dense_size(ctx->c);
    if (o->form == EG_FORM_HDG) ctx->c.ensure_hdg();
  });
}

int eg_sizes(const eg_ctx *ctx, int out[7]) {
  if (!ctx || !out) return EG_ERR_INVALID;
  const Ctx &c = ctx->c;
  const int v[7] = {c.n, c.p, c.m, c.t, c.nf, c.nu, c.nl};
  std::memcpy(out, v, sizeof v);
  return EG_OK;
}

long long eg_device_bytes(const eg_ctx *ctx) { return ctx ? ctx->c.bytes : 0; }

int eg_upload(eg_ctx *ctx, int slot, const double *src) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    size_t count = 0;
    double *dst = eg::slot_ptr(c, slot, count);
    eg::upload_vec(c, dst, src, count);
    if (slot == EG_SLOT_U || slot == EG_SLOT_OLD) c.residual_ready = false;
    c.sync();
  });
}

int eg_download(eg_ctx *ctx, int slot, double *dst) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    if (slot == EG_SLOT_X || slot == EG_SLOT_Y) {
      if (!c.XY || !c.condensed) eg::fail(EG_ERR_INVALID, "no condensation available");
      const size_t ld = (size_t)c.m * (4 * c.t + 1) * sizeof(double);
      if (slot == EG_SLOT_X) {
        const size_t w = (size_t)c.m * 4 * c.t * sizeof(double);
        EG_CUDA(cudaMemcpy2DAsync(dst, w, c.XY, ld, w, c.n, cudaMemcpyDefault, c.stream));
      } else {
        const size_t w = (size_t)c.m * sizeof(double);
        EG_CUDA(cudaMemcpy2DAsync(dst, w, c.XY + (size_t)c.m * 4 * c.t, ld, w, c.n, cudaMemcpyDefault,
                                  c.stream));
      }
      c.sync();
      return;
    }
    if (slot == EG_SLOT_PC_BLOCKS && c.opts.precond == EG_PC_BLOCK_ILU0) {
      const eg::IluPlan &P = c.ilu[c.opts.form];
      if (!P.built) eg::fail(EG_ERR_INVALID, "no preconditioner built");
      eg::download_vec(c, dst, P.data, (size_t)P.nnzb * P.B * P.B);
      return;
    }
    if (slot == EG_SLOT_PC_BLOCKS) {
      if (c.opts.form == EG_FORM_DG) {
        if (!c.pc_dg) eg::fail(EG_ERR_INVALID, "no preconditioner built");
        if (eg::dg_pc_is_record(c)) {
          // the slot holds the inverses the record applies, column-major
          if (!dst) eg::fail(EG_ERR_INVALID, "null vector");
          eg::download_dg_record_inverse(c, dst);
        } else {
          eg::download_vec(c, dst, c.pc_dg, (size_t)c.n * c.m * c.m);
        }
      } else {
        if (!c.pc_hdg) eg::fail(EG_ERR_INVALID, "no preconditioner built");
        if (!dst) eg::fail(EG_ERR_INVALID, "null vector");
        // stored row-major for the block GEMV; the slot is column-major
        eg::launch_transpose_blocks(c, c.pc_hdg, c.nf, c.t);
        eg::download_vec(c, dst, c.pc_hdg, (size_t)c.nf * c.t * c.t);
        eg::launch_transpose_blocks(c, c.pc_hdg, c.nf, c.t);
        c.sync();
      }
      return;
    }
    size_t count = 0;
    const double *src = eg::slot_ptr(c, slot, count);
    eg::download_vec(c, dst, src, count);
  });
}

int eg_initial(eg_ctx *ctx) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    eg::field_initial(c, c.u);
    c.residual_ready = false;
    c.sync();
  });
}

int eg_freeze(eg_ctx *ctx, double stage_dt, int check_admissible, double *wave_rate) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    eg::launch_freeze(c, c.u, check_admissible != 0);
    c.check_device_error();
    eg::launch_copy(c, c.nu, c.u, c.old);
    c.geo.dt = stage_dt;
    c.residual_ready = false;
    if (wave_rate) {
      EG_CUDA(cudaMemcpyAsync(c.hscal + eg::DS_WAVE, c.dscal + eg::DS_WAVE, sizeof(double),
                              cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      *wave_rate = c.hscal[eg::DS_WAVE] / std::min(c.desc.hx, c.desc.hy);
    }
    c.sync();
  });
}

int eg_set_dt(eg_ctx *ctx, double dt) {
  if (!ctx) return EG_ERR_INVALID;
  ctx->c.geo.dt = dt;
  ctx->c.residual_ready = false;
  return EG_OK;
}

int eg_residual(eg_ctx *ctx) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    eg::launch_residual(c, c.u, c.old, c.r);
    c.sync();
  });
}

int eg_cell_norm(eg_ctx *ctx, int slot, double *out) {
  if (!ctx || !out) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    size_t count = 0;
    const double *x = eg::slot_ptr(c, slot, count);
    if ((int)count != c.nu) eg::fail(EG_ERR_INVALID, "Cell norm size mismatch");
    *out = eg::cell_norm(c, x);
  });
}

int eg_admissible(eg_ctx *ctx, int slot, int *ok) {
  if (!ctx || !ok) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    size_t count = 0;
    const double *x = eg::slot_ptr(c, slot, count);
    if ((int)count != c.nu) eg::fail(EG_ERR_INVALID, "size mismatch");
    eg::launch_admissible(c, x);
    EG_CUDA(cudaMemcpyAsync(c.herr + 1, c.derr + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    *ok = c.herr[1];
  });
}

int eg_dg_apply(eg_ctx *ctx, const double *x, double *y) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    eg::upload_vec(c, c.tmp_body, x, c.nu);
    eg::launch_dg_refresh(c, c.u);
    eg::launch_dg_apply_cached(c, c.tmp_body, c.er);
    eg::download_vec(c, y, c.er, c.nu);
  });
}

int eg_condense(eg_ctx *ctx) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    eg::launch_condense(c, c.u, c.r);
    c.check_device_error();
  });
}

int eg_schur_apply(eg_ctx *ctx, const double *v, double *y) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    if (!c.condensed) eg::fail(EG_ERR_INVALID, "no condensation available");
    eg::upload_vec(c, c.tmp_trace, v, c.nl);
    eg::launch_schur_apply(c, c.tmp_trace, c.lam);
    eg::download_vec(c, y, c.lam, c.nl);
  });
}

int eg_recover(eg_ctx *ctx, const double *lam, double *du) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    if (!c.condensed) eg::fail(EG_ERR_INVALID, "no condensation available");
    eg::upload_vec(c, c.tmp_trace, lam, c.nl);
    eg::launch_recover(c, c.tmp_trace, c.du);
    eg::download_vec(c, du, c.du, c.nu);
  });
}

int eg_pc_factor(eg_ctx *ctx, int factor) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] { eg::pc_factor(ctx->c, ctx->c.opts.form, factor != 0); });
}

int eg_set_desc(eg_ctx *ctx, const eg_desc *d) {
  if (!ctx || !d) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    if (d->nx != c.desc.nx || d->ny != c.desc.ny || d->k != c.desc.k)
      eg::fail(EG_ERR_INVALID, "a context keeps its mesh size and degree");
    for (int i = 0; i < c.p; ++i)
      if (d->tensor_node[i] != i) eg::fail(EG_ERR_INVALID, "native node order must be lexicographic (x fastest)");
    eg::upload_desc(c, *d);
  });
}

int eg_pc_size(const eg_ctx *ctx, long long *count) {
  if (!ctx || !count) return EG_ERR_INVALID;
  const Ctx &c = ctx->c;
  if (c.opts.precond == EG_PC_BLOCK_ILU0) {
    const eg::IluPlan &P = c.ilu[c.opts.form];
    *count = P.built ? (long long)P.nnzb * P.B * P.B : 0;
  } else {
    *count = c.opts.form == EG_FORM_DG ? (long long)c.n * c.m * c.m : (long long)c.nf * c.t * c.t;
  }
  return EG_OK;
}

int eg_pc_apply(eg_ctx *ctx, const double *b, double *x) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    const bool ilu = c.opts.precond == EG_PC_BLOCK_ILU0;
    if (c.opts.form == EG_FORM_DG) {
      if (ilu ? !c.ilu[EG_FORM_DG].built : !c.pc_dg) eg::fail(EG_ERR_INVALID, "no preconditioner built");
      eg::upload_vec(c, c.tmp_body, b, c.nu);
      if (ilu)
        eg::launch_ilu_apply(c, EG_FORM_DG, c.tmp_body, c.er);
      else
        eg::launch_dg_jacobi_apply(c, c.tmp_body, c.er);
      c.check_device_error();
      eg::download_vec(c, x, c.er, c.nu);
    } else {
      if (ilu ? !c.ilu[EG_FORM_HDG].built : !c.pc_hdg) eg::fail(EG_ERR_INVALID, "no preconditioner built");
      c.ensure_hdg();
      eg::upload_vec(c, c.tmp_trace, b, c.nl);
      if (ilu)
        eg::launch_ilu_apply(c, EG_FORM_HDG, c.tmp_trace, c.lam);
      else
        eg::launch_block_inverse_apply(c, c.pc_hdg, c.nf, c.t, c.tmp_trace, c.lam);
      c.check_device_error();
      eg::download_vec(c, x, c.lam, c.nl);
    }
  });
}

int eg_linear_solve(eg_ctx *ctx, const double *rhs, double *x, double *eq_residual, int refresh,
                    double linear_tol, eg_linear_stats *st) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    const int form = c.opts.form;
    const int N = form == EG_FORM_DG ? c.nu : c.nl;
    double *drhs = form == EG_FORM_DG ? c.tmp_body : c.rhs;
    double *dx = form == EG_FORM_DG ? c.du : c.lam;
    double *deq = form == EG_FORM_DG ? c.er : c.tmp_trace;
    eg::upload_vec(c, drhs, rhs, N);
    if (!refresh) eg::upload_vec(c, dx, x, N);
    eg::LinearOut out;
    eg::linear_solve(c, form, drhs, dx, deq, refresh != 0, linear_tol, out);
    eg::download_vec(c, x, dx, N);
    if (eq_residual) eg::download_vec(c, eq_residual, deq, N);
    if (st) {
      st->count = out.count;
      st->residual = out.residual;
      st->rhs_norm = out.rhs_norm;
    }
  });
}

int eg_stage_begin(eg_ctx *ctx, double stage_dt) {
  if (!ctx) return EG_ERR_INVALID;
  ctx->c.geo.dt = stage_dt;
  ctx->c.residual_ready = false;
  return EG_OK;
}

int eg_newton_residual(eg_ctx *ctx, double *residual_norm) {
  if (!ctx || !residual_norm) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    const double t0 = eg::now_s();
    eg::open_update_timer(c);
    if (!c.residual_ready) eg::launch_residual(c, c.u, c.old, c.r);
    *residual_norm = eg::cell_norm(c, c.r);
    c.last_residual_s = eg::now_s() - t0;
  });
}

int eg_newton_update(eg_ctx *ctx, double residual_norm, double old_norm, eg_update_stats *st) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] { eg::newton_update(ctx->c, residual_norm, old_norm, st); });
}

int eg_integral(eg_ctx *ctx, double out[4]) {
  if (!ctx || !out) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    eg::field_integral(ctx->c, ctx->c.u, out);
  });
}

int eg_errors(eg_ctx *ctx, double time, double out[4]) {
  if (!ctx || !out) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    eg::field_errors(ctx->c, ctx->c.u, time, out);
  });
}

int eg_state_differences(eg_ctx *ctx, const double *v, double out[4]) {
  if (!ctx || !v || !out) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    Ctx &c = ctx->c;
    eg::upload_vec(c, c.tmp_body, v, c.nu);
    eg::field_differences(c, c.u, c.tmp_body, out);
  });
}

int eg_set_ilu_wait(eg_ctx *ctx, unsigned long long limit_ns, int starve) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    ctx->c.ilu_wait_limit_ns = limit_ns ? limit_ns : eg::kIluWaitLimitNs;
    ctx->c.ilu_starve = starve != 0;
    for (auto &P : ctx->c.ilu) {
      P.wait_limit_ns = ctx->c.ilu_wait_limit_ns;
      P.starve = ctx->c.ilu_starve;
    }
  });
}

int eg_profile_enable(eg_ctx *ctx, int on) {
  if (!ctx) return EG_ERR_INVALID;
  ctx->c.prof.on = on != 0;
  return EG_OK;
}
int eg_profile_reset(eg_ctx *ctx) {
  if (!ctx) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    ctx->c.sync();
    ctx->c.prof_resolve();
    for (int i = 0; i < EG_K_COUNT; ++i) {
      ctx->c.prof.ms[i] = 0.;
      ctx->c.prof.count[i] = 0;
    }
  });
}
int eg_profile_query(eg_ctx *ctx, int kernel_class, double *ms, long long *launches) {
  if (!ctx || kernel_class < 0 || kernel_class >= EG_K_COUNT) return EG_ERR_INVALID;
  return guard(ctx, [&] {
    ctx->c.sync();
    ctx->c.prof_resolve();
    if (ms) *ms = ctx->c.prof.ms[kernel_class];
    if (launches) *launches = ctx->c.prof.count[kernel_class];
  });
}
long long eg_launch_count(const eg_ctx *ctx) { return ctx ? ctx->c.launches : 0; }

int eg_differences(const eg_desc *d, const double *u, const double *v, double out[4]) {
  if (!d || !u || !v || !out) return EG_ERR_INVALID;
  try {
    eg::host::differences(*d, u, v, out);
  } catch (const std::exception &) {
    return EG_ERR_INVALID;
  }
  return EG_OK;
}

int eg_save_solution(const eg_desc *d, const double *u, const char *prefix) {
  if (!d || !u || !prefix || d->k < 0 || d->k > 8 || d->nx < 2 || d->ny < 2 || !(d->lx > 0) ||
      !(d->ly > 0))
    return EG_ERR_INVALID;
  try {
    if (!eg::host::save_solution(*d, u, prefix)) {
      g_create_error = "Cannot open solution output";
      return EG_ERR_INVALID;
    }
  } catch (const std::exception &) {
    return EG_ERR_INVALID;
  }
  return EG_OK;
}

}  // extern "C"
