// euler2d -- drop-in command line of the reference solver (src/main.cpp,
// src/options.cpp) whose Newton updates run on the GPU through the C-ABI in
// include/euler2d_cuda.h. Flags, validation messages and the CSV files
// (_iterations, _summary, _comparison, _coefficients) follow the reference;
// --device and --precision are additions (the reference binary is the CPU
// path, so --device cpu is rejected here).
#include <cmath>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/euler2d_cuda.h"

namespace {
constexpr double kPi = 3.141592653589793238462643383279502884;

void require(bool ok, const std::string &msg) {
  if (!ok) throw std::runtime_error(msg);
}

struct Options {
  int nx = 100, ny = 100, k = 1, volume_order = -1, max_newton = 30;
  int restart = 20, max_krylov = 1500, newton_steps = -1, steps = -1;
  double alpha = 45, dt = .001, end = .2, cfl = -1, safety = 1.1, tol = 1e-12, linear_tol = 1e-12;
  std::string assembly = "partial";
  std::string form = "both", solver = "gmres", precond = "block-jacobi", integrator = "ssp-dirk3",
              output = "code_test/results/run";
  bool matrix_free = true, verify = false, save_solution = true, hdg_first = false;
  bool check_update = false, timing_only = false;
  std::string ilu_ordering = "none";
  std::string device = "cuda", precision = "fp64";
};

// Restates euler::ParseOptions (src/options.cpp:8-149).
Options parse(int argc, char **argv) {
  Options o;
  bool assembly_selected = false, requested_matrix_free = false;
  for (int i = 1; i < argc; i++) {
    const std::string s = argv[i];
    auto value = [&]() {
      require(i + 1 < argc, "Missing option value");
      return std::string(argv[++i]);
    };
    if (s == "--hdg-first") {
      o.hdg_first = true;
    } else if (s == "--nx") {
      o.nx = std::stoi(value());
    } else if (s == "--ny") {
      o.ny = std::stoi(value());
    } else if (s == "--k") {
      o.k = std::stoi(value());
    } else if (s == "--cfl") {
      o.cfl = std::stod(value());
      require(o.cfl > 0, "--cfl must be positive");
    } else if (s == "--steps") {
      o.steps = std::stoi(value());
      require(o.steps > 0, "--steps must be positive");
    } else if (s == "--newton-steps") {
      o.newton_steps = std::stoi(value());
      require(o.newton_steps > 0, "--newton-steps must be positive");
    } else if (s == "--check-update") {
      o.check_update = true;
    } else if (s == "--timing-only") {
      o.timing_only = true;
    } else if (s == "--ilu-ordering") {
      o.ilu_ordering = value();
    } else if (s == "--dt") {
      o.dt = std::stod(value());
    } else if (s == "--T") {
      o.end = std::stod(value());
    } else if (s == "--alpha-deg") {
      o.alpha = std::stod(value());
    } else if (s == "--safety") {
      o.safety = std::stod(value());
    } else if (s == "--volume-order") {
      o.volume_order = std::stoi(value());
    } else if (s == "--assembly") {
      o.assembly = value();
      assembly_selected = true;
    } else if (s == "--form") {
      o.form = value();
    } else if (s == "--solver") {
      o.solver = value();
    } else if (s == "--integrator") {
      o.integrator = value();
    } else if (s == "--precond") {
      o.precond = value();
    } else if (s == "--output") {
      o.output = value();
    } else if (s == "--matrix-free") {
      requested_matrix_free = true;
    } else if (s == "--no-save-solution") {
      o.save_solution = false;
    } else if (s == "--linear-tol") {
      o.linear_tol = std::stod(value());
    } else if (s == "--newton-tol") {
      o.tol = std::stod(value());
    } else if (s == "--restart") {
      o.restart = std::stoi(value());
    } else if (s == "--max-krylov") {
      o.max_krylov = std::stoi(value());
    } else if (s == "--max-newton") {
      o.max_newton = std::stoi(value());
    } else if (s == "--verify") {
      o.verify = true;
    } else if (s == "--device") {
      o.device = value();
    } else if (s == "--precision") {
      o.precision = value();
    } else if (s == "--help") {
      std::cout << "--nx N --ny N --k 0..8 --alpha-deg A (default 45)\n"
                   "--dt DT | --cfl C (CFL wins; h=min(hx,hy), speed includes safety)\n"
                   "--T T (default .2) | --steps N (steps wins; no T clipping)\n"
                   "--max-newton N --newton-tol E | --newton-steps N (fixed updates/stage)\n"
                   "--form dg|hdg|both --integrator ssp-dirk3|be\n"
                   "--solver gmres\n"
                   "--precond block-jacobi|block-ilu0 --ilu-ordering none\n"
                   "--assembly full|element|partial --matrix-free --safety 1.1\n"
                   "--linear-tol E --restart N --max-krylov N --output PREFIX\n"
                   "--check-update --timing-only --no-save-solution --hdg-first\n"
                   "--device cuda --precision fp64|mixed\n";
      std::exit(EXIT_SUCCESS);
    } else {
      throw std::runtime_error("Unknown option: " + s);
    }
  }
  require(o.nx >= 2 && o.ny >= 2 && o.k >= 0 && o.k <= 8 && o.dt > 0 && o.end >= 0 && o.safety >= 1 &&
              o.tol > 0 && o.linear_tol > 0,
          "Invalid mesh, degree, time or safety");
  const long double cells = static_cast<long double>(o.nx) * o.ny, q = o.k + 1.L;
  require(4 * cells * q * q <= std::numeric_limits<int>::max() &&
              8 * cells * q <= std::numeric_limits<int>::max(),
          "Mesh/degree exceeds MFEM int DOF capacity");
  require(std::isfinite(o.alpha) && std::isfinite(o.dt) && std::isfinite(o.end) &&
              std::isfinite(o.safety) && std::isfinite(o.tol) && std::isfinite(o.linear_tol),
          "Nonfinite option");
  require(o.form == "dg" || o.form == "hdg" || o.form == "both", "Invalid form");
  require(o.integrator == "ssp-dirk3" || o.integrator == "be", "Invalid time integrator");
  require(o.solver == "gmres" || o.solver == "direct" || o.solver == "dense", "Invalid solver");
  require(o.restart > 0 && o.max_krylov > 0 && o.max_newton > 0, "Iteration limits must be positive");
  require((o.cfl == -1 || (std::isfinite(o.cfl) && o.cfl > 0)) && (o.steps == -1 || o.steps > 0) &&
              (o.newton_steps == -1 || o.newton_steps > 0),
          "CFL, steps and fixed Newton updates must be positive when supplied");
  require(o.alpha > 0 && o.alpha < 90, "Require 0 < alpha-deg < 90");
  const double angle = o.alpha * kPi / 180;
  require(std::isfinite(2 / std::cos(angle)) && std::isfinite(2 / std::sin(angle)),
          "Angle produces nonfinite domain lengths");
  require(o.ilu_ordering == "none" || o.ilu_ordering == "mdf", "Invalid ILU ordering");
  require(o.volume_order == -1 || o.volume_order == 2 * o.k + 1,
          "Volume rule must be (k+1)^2 GL points (order 2k+1)");
  o.volume_order = -1;
  if (o.solver == "gmres") {
    require(o.precond == "block-jacobi" || o.precond == "block-ilu0", "Invalid preconditioner");
    if (requested_matrix_free) o.assembly = "partial";
    o.matrix_free = o.assembly != "full";
  } else {
    require(!requested_matrix_free, "Direct LU requires an assembled matrix");
    if (!assembly_selected) o.assembly = "full";
    require(o.assembly == "full", "Direct LU requires --assembly full");
    o.matrix_free = false;
    o.precond = "none";
  }
  require(o.assembly == "full" || o.assembly == "element" || o.assembly == "partial", "Invalid assembly");
  if (o.timing_only) o.save_solution = false;
  // Device-path scope (the reference binary serves the rest).
  require(o.device == "cuda", "This executable is the --device cuda path; use the reference euler2d for CPU runs");
  require(o.precision == "fp64" || o.precision == "mixed", "Invalid precision");
  // --solver direct is MKL PARDISO, which the reference's portable build lacks too
  require(o.solver != "direct", "--solver direct requires MFEM with MKL PARDISO");
  require(o.precision == "fp64" || o.assembly != "full", "--precision mixed requires --assembly partial or element");
  require(o.ilu_ordering == "none", "--ilu-ordering mdf is not available with --device cuda");
  require(!o.verify, "--verify is a CPU diagnostic of the reference build");
  return o;
}

void check(int rc, eg_ctx *ctx) {
  if (rc != EG_OK) {
    std::string msg = eg_last_error(ctx);
    if (msg.empty()) msg = eg_status_string(rc);
    throw std::runtime_error(msg);
  }
}

struct FormResult {
  std::vector<double> u;
  eg_run_result r{};
};

FormResult run_form(const Options &o, const eg_desc &desc, const std::string &form) {
  eg_opts eo;
  eg_opts_default(&eo);
  eo.form = form == "dg" ? EG_FORM_DG : EG_FORM_HDG;
  eo.precond = o.precond == "block-ilu0" ? EG_PC_BLOCK_ILU0 : EG_PC_BLOCK_JACOBI;
  eo.assembly = o.assembly == "full" ? EG_ASSEMBLY_FULL
                : o.assembly == "element" ? EG_ASSEMBLY_ELEMENT : EG_ASSEMBLY_PARTIAL;
  eo.precision = o.precision == "mixed" ? EG_PRECISION_MIXED : EG_PRECISION_FP64;
  eo.restart = o.restart;
  eo.max_krylov = o.max_krylov;
  eo.linear_tol = o.linear_tol;
  eo.check_update = o.check_update ? 1 : 0;
  eo.solver = o.solver == "dense" ? EG_SOLVER_DENSE : EG_SOLVER_GMRES;
  eg_ctx *ctx = nullptr;
  check(eg_create(&desc, &eo, &ctx), ctx);
  const std::string prefix = o.output + "_" + form;
  eg_run_opts ro{};
  ro.integrator = o.integrator == "be" ? 1 : 0;
  ro.steps = o.steps;
  ro.newton_steps = o.newton_steps;
  ro.max_newton = o.max_newton;
  ro.dt = o.dt;
  ro.cfl = o.cfl;
  ro.end = o.end;
  ro.tol = o.tol;
  ro.timing_only = o.timing_only;
  ro.save_solution = o.save_solution;
  ro.prefix = prefix.c_str();
  ro.form_name = form.c_str();
  ro.assembly_name = o.assembly.c_str();
  ro.solver_name = o.solver.c_str();
  ro.precond_name = o.precond.c_str();
  ro.ilu_ordering_name = o.ilu_ordering.c_str();
  ro.check_update = o.check_update;
  FormResult out;
  int rc = eg_run(ctx, &ro, &out.r);
  if (rc == EG_OK) {
    int sizes[7];
    eg_sizes(ctx, sizes);
    out.u.resize(sizes[5]);
    rc = eg_download(ctx, EG_SLOT_U, out.u.data());
  }
  std::string msg = rc != EG_OK ? std::string(eg_last_error(ctx)) : std::string();
  eg_destroy(ctx);
  if (rc != EG_OK) throw std::runtime_error(msg.empty() ? eg_status_string(rc) : msg);
  return out;
}
}  // namespace

int main(int argc, char **argv) {
  try {
    Options o = parse(argc, argv);
    const double gamma = 3.;  // the simple-wave problem's gamma (src/main.cpp:8)
    const auto parent = std::filesystem::path(o.output).parent_path();
    if (!parent.empty()) std::filesystem::create_directories(parent);
    require(o.steps > 0 || o.end < 4 / ((gamma + 1) * kPi), "Exact solution requires T < 4/((gamma+1)*pi)");
    eg_desc desc;
    require(eg_desc_simple_wave(&desc, o.nx, o.ny, o.k, o.alpha, gamma, o.safety) == EG_OK,
            "Invalid mesh, degree, time or safety");
    FormResult dg, hdg;
    if (o.form == "both" && o.hdg_first) {
      hdg = run_form(o, desc, "hdg");
      dg = run_form(o, desc, "dg");
    } else {
      if (o.form != "hdg") dg = run_form(o, desc, "dg");
      if (o.form != "dg") hdg = run_form(o, desc, "hdg");
    }
    if (o.form == "both") {
      double diff = 0.;
      for (size_t i = 0; i < dg.u.size(); ++i) diff = std::max(diff, std::abs(dg.u[i] - hdg.u[i]));
      double l2[4];
      eg_differences(&desc, dg.u.data(), hdg.u.data(), l2);
      double combined = 0.;
      for (double v : l2) combined += v * v;
      combined = std::sqrt(combined);
      std::ofstream f(o.output + "_comparison.csv");
      f << "max_nodal_difference,rho_L2_difference,rhou_L2_difference,"
           "rhov_L2_difference,energy_L2_difference,solution_L2_difference,"
           "dg_over_hdg_mean_newton\n"
        << std::setprecision(17) << diff << ',' << l2[0] << ',' << l2[1] << ',' << l2[2] << ','
        << l2[3] << ',' << combined << ','
        << (dg.r.updates && hdg.r.updates && hdg.r.newton_seconds > 0
                ? (dg.r.newton_seconds / dg.r.updates) / (hdg.r.newton_seconds / hdg.r.updates)
                : 0.)
        << '\n';
      std::cout << "DG/HDG max nodal difference=" << diff << '\n';
      require(diff < 1e-7, "DG/HDG final solutions disagree");
    }
    return 0;
  } catch (const std::exception &e) {
    std::cerr << "ERROR: " << e.what() << '\n';
    return 1;
  }
}
