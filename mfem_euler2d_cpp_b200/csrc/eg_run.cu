// Time loop of the reference (euler::Run, src/stepper.cpp:28-292) driving the
// device Newton update: SSP-DIRK3 (or backward Euler) stages, beginning-of-
// step Freeze + CFL step, per-stage Freeze, Newton loop with the reference's
// convergence test, stage slopes and the DIRK combination. Writes the same
// _iterations.csv / _summary.csv columns. The loop is a resumable state
// machine so a benchmark can advance it one accepted Newton update at a time.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>

#include "eg_internal.h"
#include "eg_setup.h"

struct eg_ctx {
  eg::Ctx c;
};

namespace eg {

static double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static constexpr double kPi = 3.141592653589793238462643383279502884;

// SSP-DIRK3(4,3,3) tableau (src/stepper.cpp:71-80)
static constexpr double kAlpha = 0.24169426078821;
static constexpr double kBeta = kAlpha / 4.;
static constexpr double kEta = 0.12915286960590;
static const double kA[4][4] = {{kAlpha, 0., 0., 0.},
                                {-kAlpha, kAlpha, 0., 0.},
                                {0., 1. - kAlpha, kAlpha, 0.},
                                {kBeta, kEta, .5 - kBeta - kEta - kAlpha, kAlpha}};
static const double kB[4] = {0., 1. / 6., 1. / 6., 2. / 3.};
static const double kC[4] = {kAlpha, 0., 1., .5};

__global__ void add_scaled_kernel(int N, double a, const double *__restrict__ x, double *__restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}
// slope = (u - base) * s
__global__ void slope_kernel(int N, const double *__restrict__ u, const double *__restrict__ base,
                             double s, double *__restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    out[i] = (u[i] - base[i]) * s;
}

struct Stepper {
  Ctx &c;
  eg_run_opts ro{};
  std::string prefix, form_name, assembly, solver, precond, ordering;
  double *step_state = nullptr, *stage_base = nullptr, *slope[4] = {nullptr, nullptr, nullptr, nullptr};
  int stage_count = 4;
  int step = 0, stage = 0, it = 0, limit = 0;
  double time = 0., dt = 0., rate = 0., dt_sum = 0., max_cfl = 0.;
  double stage_dt = 0., physical_scale = 0., old_norm = 0., r0 = -1.;
  bool final_step = false, converged = false, done = false;
  double initial_integral[4] = {0, 0, 0, 0};
  // last update, for logging
  double last_rms = 0.;
  int last_it = 0;

  explicit Stepper(Ctx &ctx) : c(ctx) {}

  bool keep_stepping() const { return ro.steps > 0 ? step < ro.steps : !final_step; }

  void grid_add(double a, const double *x, double *y) {
    ProfScope ps(c, EG_K_VECTOR, 1);
    add_scaled_kernel<<<std::min((c.nu + 255) / 256, 148 * 16), 256, 0, c.stream>>>(c.nu, a, x, y);
    EG_CUDA(cudaGetLastError());
  }

  void begin() {
    if (!c.step_bufs) c.step_bufs = c.alloc_n<double>((size_t)6 * c.nu);  // kept for later schedules
    int slot = 0;
    for (double **v : {&step_state, &stage_base, &slope[0], &slope[1], &slope[2], &slope[3]}) {
      *v = c.step_bufs + (size_t)(slot++) * c.nu;
      EG_CUDA(cudaMemsetAsync(*v, 0, sizeof(double) * c.nu, c.stream));
    }
    field_initial(c, c.u);  // Problem::Initial on the device
    launch_admissible(c, c.u);
    EG_CUDA(cudaMemcpyAsync(c.herr + 1, c.derr + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (!c.herr[1]) fail(EG_ERR_INITIAL, "Initial projection not positive; refine mesh");
    field_integral(c, c.u, initial_integral);
    stage_count = ro.integrator == 1 ? 1 : 4;
    final_step = time >= ro.end;
    if (keep_stepping())
      begin_step();
    else
      done = true;
  }

  void freeze_at_u(double stage_step) {
    launch_freeze(c, c.u, false);
    c.check_device_error();
    launch_copy(c, c.nu, c.u, c.old);
    c.geo.dt = stage_step;
  }

  void begin_step() {
    launch_copy(c, c.nu, c.u, step_state);
    freeze_at_u(ro.dt);
    EG_CUDA(cudaMemcpyAsync(c.hscal + DS_WAVE, c.dscal + DS_WAVE, sizeof(double), cudaMemcpyDeviceToHost,
                            c.stream));
    c.sync();
    rate = c.hscal[DS_WAVE] / std::min(c.desc.hx, c.desc.hy);
    dt = ro.cfl > 0 ? ro.cfl / rate : ro.dt;
    if (ro.steps < 0) {
      final_step = time + dt >= ro.end;
      if (final_step) dt = ro.end - time;
    }
    if (!(std::isfinite(dt) && dt > 0 && time + dt < 4 / ((c.desc.gamma + 1) * kPi)))
      fail(EG_ERR_STEP_INTERVAL, "Step leaves the smooth simple-wave interval T < 4/((gamma+1)*pi)");
    stage = 0;
    begin_stage();
  }

  void begin_stage() {
    const double diag = ro.integrator == 1 ? 1. : kA[stage][stage];
    launch_copy(c, c.nu, step_state, stage_base);
    if (ro.integrator != 1)
      for (int j = 0; j < stage; ++j) grid_add(dt * kA[stage][j], slope[j], stage_base);
    if (stage > 0) freeze_at_u(diag * dt);
    stage_dt = diag * dt;
    c.geo.dt = stage_dt;
    launch_copy(c, c.nu, stage_base, c.old);
    physical_scale = 1 / (stage_dt * std::sqrt(c.desc.lx * c.desc.ly));
    old_norm = cell_norm(c, stage_base);
    r0 = -1.;
    converged = false;
    c.residual_ready = false;
    limit = ro.newton_steps > 0 ? ro.newton_steps : ro.max_newton;
    it = 0;
  }

  void end_stage() {
    if (!(converged || ro.newton_steps > 0)) fail(EG_ERR_NEWTON_CONVERGE, "Newton failed to converge");
    c.launches += 1;
    slope_kernel<<<std::min((c.nu + 255) / 256, 148 * 16), 256, 0, c.stream>>>(c.nu, c.u, stage_base,
                                                                             1. / stage_dt, slope[stage]);
    EG_CUDA(cudaGetLastError());
    ++stage;
    if (stage < stage_count) {
      begin_stage();
      return;
    }
    if (ro.integrator != 1) {
      launch_copy(c, c.nu, step_state, c.u);
      for (int s = 0; s < 4; ++s) grid_add(dt * kB[s], slope[s], c.u);
      c.residual_ready = false;
      launch_admissible(c, c.u);
      EG_CUDA(cudaMemcpyAsync(c.herr + 1, c.derr + 1, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      if (!c.herr[1]) fail(EG_ERR_DIRK_INADMISSIBLE, "SSP-DIRK3 step produced an inadmissible state");
    }
    time = ro.steps < 0 && final_step ? ro.end : time + dt;
    dt_sum += dt;
    max_cfl = std::max(max_cfl, rate * dt);
    ++step;
    if (keep_stepping())
      begin_step();
    else
      done = true;
  }

  // Advance to and perform the next accepted Newton update. Returns false when
  // the schedule is finished.
  bool next(eg_update_stats *st) {
    while (!done) {
      double rn = 0.;
      {
        const double t0 = wall_s();
        EG_CUDA(cudaEventRecord(c.ev0, c.stream));
        c.update_timer_open = true;
        if (!c.residual_ready) launch_residual(c, c.u, c.old, c.r);
        rn = cell_norm(c, c.r);
        c.last_residual_s = wall_s() - t0;
      }
      const double rms = physical_scale * rn;
      if (r0 < 0) r0 = rms;
      if (ro.newton_steps < 0 && rms <= ro.tol * std::max(1., r0)) {
        converged = true;
        c.update_timer_open = false;
        end_stage();
        continue;
      }
      if (it == limit) {
        c.update_timer_open = false;
        end_stage();
        continue;
      }
      eg_update_stats s{};
      newton_update(c, rn, old_norm, &s);
      last_rms = rms;
      last_it = it;
      ++it;
      if (st) *st = s;
      return true;
    }
    return false;
  }
};

}  // namespace eg

struct eg_stepper {
  eg::Stepper s;
  explicit eg_stepper(eg::Ctx &c) : s(c) {}
};

template <class F>
static int guard_run(eg::Ctx &c, F &&f) {
  if (c.broken) {
    c.err = eg_status_string(EG_ERR_CONTEXT_LOST);
    return EG_ERR_CONTEXT_LOST;
  }
  try {
    f();
    return EG_OK;
  } catch (const eg::Failure &e) {
    c.err = e.msg;
    return e.status;
  } catch (const std::exception &e) {
    c.err = e.what();
    return EG_ERR_INVALID;
  }
}

static void copy_run_opts(eg::Stepper &s, const eg_run_opts *ro) {
  s.ro = *ro;
  s.prefix = ro->prefix ? ro->prefix : "run";
  s.form_name = ro->form_name ? ro->form_name : (s.c.opts.form == EG_FORM_DG ? "dg" : "hdg");
  s.assembly = ro->assembly_name ? ro->assembly_name : "partial";
  s.solver = ro->solver_name ? ro->solver_name : "gmres";
  s.precond = ro->precond_name ? ro->precond_name
                               : (s.c.opts.precond == EG_PC_BLOCK_JACOBI ? "block-jacobi" : "block-ilu0");
  s.ordering = ro->ilu_ordering_name ? ro->ilu_ordering_name : "none";
}

extern "C" {

int eg_stepper_create(eg_ctx *ctx, const eg_run_opts *ro, eg_stepper **out) {
  if (!ctx || !ro || !out) return EG_ERR_INVALID;
  *out = nullptr;
  auto *st = new eg_stepper(ctx->c);
  copy_run_opts(st->s, ro);
  const int rc = guard_run(ctx->c, [&] { st->s.begin(); });
  if (rc != EG_OK) {
    delete st;
    return rc;
  }
  *out = st;
  return EG_OK;
}

int eg_stepper_next(eg_stepper *s, eg_update_stats *st) {
  if (!s) return EG_ERR_INVALID;
  bool more = false;
  const int rc = guard_run(s->s.c, [&] { more = s->s.next(st); });
  if (rc != EG_OK) return rc;
  return more ? EG_OK : -1;
}

void eg_stepper_destroy(eg_stepper *s) { delete s; }

int eg_stepper_finish(eg_stepper *s, eg_run_result *res) {
  if (!s || !res) return EG_ERR_INVALID;
  eg::Stepper &st = s->s;
  eg::Ctx &c = st.c;
  return guard_run(c, [&] {
    if (!st.done) eg::fail(EG_ERR_INVALID, "schedule not finished");
    eg_run_result out{};
    out.final_time = st.time;
    out.time_steps = st.step;
    // errors and integrals on the device: the state stays resident
    eg::field_errors(c, c.u, st.time, out.errors);
    double fin[4];
    eg::field_integral(c, c.u, fin);
    for (int k = 0; k < 4; ++k) out.drift = std::max(out.drift, std::abs(fin[k] - st.initial_integral[k]));
    *res = out;
  });
}

int eg_run(eg_ctx *ctx, const eg_run_opts *ro, eg_run_result *res) {
  if (!ctx || !ro) return EG_ERR_INVALID;
  eg::Ctx &c = ctx->c;
  eg::Stepper s(c);
  copy_run_opts(s, ro);
  eg_run_result out{};
  const int rc = guard_run(c, [&] {
    std::ofstream log;
    if (!ro->timing_only) {
      log.open(s.prefix + "_iterations.csv");
      if (!log) eg::fail(EG_ERR_INVALID, "Cannot open iteration output");
      log << "form,matrix_free,step,stage,newton,time,stage_time,dt,cfl,"
             "residual_physical_rms,damping,"
             "krylov_iterations,linear_relative_residual,dg_linear_relative_residual,"
             "residual_s,validation_s,jacobian_s,condensation_s,assembly_s,setup_s,"
             "solve_s,recovery_s,line_search_s,iteration_s,update_check_relative\n"
          << std::setprecision(17);
    }
    const double begin = eg::wall_s();
    s.begin();
    eg_update_stats st{};
    const int matrix_free = c.opts.assembly == EG_ASSEMBLY_FULL ? 0 : 1;
    while (true) {
      // capture schedule position before next() may roll the stage forward
      bool more = s.next(&st);
      if (!more) break;
      ++out.updates;
      out.newton_seconds += st.iteration_s;
      out.newton_device_ms += st.device_ms;
      if (log.is_open()) {
        const double stage_time = s.time + (ro->integrator == 1 ? 1. : eg::kC[s.stage]) * s.dt;
        log << s.form_name << ',' << matrix_free << ',' << s.step << ',' << s.stage << ',' << s.last_it
            << ',' << s.time + s.dt << ',' << stage_time << ',' << s.dt << ',' << s.rate * s.dt << ','
            << s.last_rms << ',' << st.damping << ',' << st.krylov_iterations << ','
            << st.linear_relative_residual << ',' << st.dg_linear_relative_residual << ','
            << st.residual_s << ',' << st.validation_s << ',' << st.jacobian_s << ','
            << st.condensation_s << ',' << st.assembly_s << ',' << st.setup_s << ',' << st.solve_s
            << ',' << st.recovery_s << ',' << st.line_search_s << ',' << st.iteration_s << ','
            << st.update_check << '\n';
      }
    }
    out.seconds = eg::wall_s() - begin;
    out.final_time = s.time;
    out.time_steps = s.step;
    eg::field_errors(c, c.u, s.time, out.errors);
    double fin[4];
    eg::field_integral(c, c.u, fin);
    for (int k = 0; k < 4; ++k) out.drift = std::max(out.drift, std::abs(fin[k] - s.initial_integral[k]));
    if (ro->save_solution) {
      std::vector<double> u(c.nu);
      EG_CUDA(cudaMemcpyAsync(u.data(), c.u, sizeof(double) * c.nu, cudaMemcpyDeviceToHost, c.stream));
      c.sync();
      if (!eg::host::save_solution(c.desc, u.data(), s.prefix))
        eg::fail(EG_ERR_INVALID, "Cannot open solution output");
    }
    std::ofstream summary(s.prefix + "_summary.csv");
    if (!summary) eg::fail(EG_ERR_INVALID, "Cannot open summary output");
    summary << "form,nx,ny,k,gamma,integrator,stages,T,dt,cfl,"
               "actual_max_cfl,mean_dt,"
               "volume_dofs,trace_dofs,matrix_free,assembly,solver,preconditioner,"
               "ilu_ordering,requested_steps,fixed_newton_steps,time_steps,"
               "newton_updates,newton_s,mean_newton_s,time_loop_s,rho_L2,rhou_L2,"
               "rhov_L2,energy_L2,max_conservation_drift,check_update,device,precision,"
               "newton_device_s,mean_newton_device_s\n"
            << std::setprecision(17);
    const double mean = out.updates ? out.newton_seconds / out.updates : 0.;
    out.mean_newton_s = mean;
    const double dev_s = out.newton_device_ms * 1e-3;
    summary << s.form_name << ',' << c.desc.nx << ',' << c.desc.ny << ',' << c.desc.k << ','
            << c.desc.gamma << ',' << (ro->integrator == 1 ? "be" : "ssp-dirk3") << ','
            << (ro->integrator == 1 ? 1 : 4) << ',' << s.time << ',' << ro->dt << ',' << ro->cfl << ','
            << s.max_cfl << ',' << (s.step ? s.dt_sum / s.step : 0.) << ',' << c.nu << ',' << c.nl << ','
            << matrix_free << ',' << s.assembly << ',' << s.solver << ',' << s.precond << ','
            << s.ordering << ',' << ro->steps << ',' << ro->newton_steps << ',' << s.step << ','
            << out.updates << ',' << out.newton_seconds << ',' << mean << ',' << out.seconds;
    for (double x : out.errors) summary << ',' << x;
    summary << ',' << out.drift << ',' << ro->check_update << ",cuda,"
            << (c.opts.precision == EG_PRECISION_MIXED ? "mixed" : "fp64") << ',' << dev_s << ','
            << (out.updates ? dev_s / out.updates : 0.) << '\n';
    std::cout << s.form_name << " k=" << c.desc.k << " " << c.desc.nx << "x" << c.desc.ny
              << " updates=" << out.updates << " mean_newton_s=" << mean << " rho_L2=" << out.errors[0]
              << " drift=" << out.drift << '\n';
  });
  if (res) *res = out;
  return rc;
}

}  // extern "C"
