/*
 * euler2d_cuda.h -- C-ABI of the B200 (sm_100a) Newton-update engine for the
 * frozen-HLL DG / condensed-HDG 2-D Euler solver of YueWu2002/mfem_euler2d_cpp.
 *
 * The reference has no FFI; its seams are C++ classes in include/euler.hpp.
 * Every entry point below names the reference function it replaces, so a
 * maintainer can route `--device cuda` through this library from the
 * reference's Run() (src/stepper.cpp:28) without touching its CPU path.
 *
 * Conventions
 *  - Every call returns an int status: EG_OK (0) or one of the EG_ERR_* codes,
 *    which map 1:1 to the reference's require() messages (eg_status_string()).
 *    No C++ exception, device trap or unbounded wait crosses this boundary.
 *  - A context owns all device memory of one problem instance and one CUDA
 *    stream; it is not thread-safe. Separate contexts are independent.
 *  - Vector arguments may be host or device pointers (the library copies with
 *    unified addressing). Layouts are the reference's (include/euler.hpp:44-45):
 *    body  u[e*m + 4*i + c]  (cell e, native GL node i, component c),
 *    trace l[f*t + 4*j + c]  (periodic face f, face GL node j, component c),
 *    with q = k+1, p = q*q, m = 4p, t = 4q, n = nx*ny, nf = 2n.
 *  - Cells are numbered row-major (e = iy*nx + ix); face 2e is the x-face
 *    between e and its +x neighbour, face 2e+1 the y-face between e and its
 *    +y neighbour (src/problem.cpp:77-90).
 */
#ifndef EULER2D_CUDA_H
#define EULER2D_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define EG_MAX_Q 9 /* k <= 8 (src/options.cpp:97) */
#define EG_MAX_P (EG_MAX_Q * EG_MAX_Q)

/* ------------------------------------------------------------ status codes */
enum eg_status {
  EG_OK = 0,
  EG_ERR_INVALID = 1,           /* invalid argument or unsupported configuration */
  EG_ERR_CUDA = 2,              /* CUDA runtime failure (text in eg_last_error) */
  EG_ERR_NONPOSITIVE_FACE = 3,  /* "Nonpositive old face state; refine mesh" physics.cpp:46-49 */
  EG_ERR_ROE_SOUND = 4,         /* "Invalid Roe sound speed" physics.cpp:58 */
  EG_ERR_DEGENERATE_HLL = 5,    /* "Degenerate HLL speeds" problem.cpp:369 */
  EG_ERR_INADMISSIBLE = 6,      /* "Old state is inadmissible; refine mesh" problem.cpp:353 */
  EG_ERR_SINGULAR_CELL = 7,     /* "Singular streaming HDG cell factor" condensation.cpp:137 */
  EG_ERR_SINGULAR_JACOBI = 8,   /* "Singular block Jacobi factor" linear.cpp:201 */
  EG_ERR_SINGULAR_ILU = 9,      /* "Singular BSR ILU diagonal" block_ilu.cpp:84 */
  EG_ERR_GMRES_BREAKDOWN = 10,  /* "GMRES Arnoldi breakdown" linear.cpp:129 */
  EG_ERR_GMRES_NONFINITE = 11,  /* "Nonfinite GMRES residual" linear.cpp:152 */
  EG_ERR_GMRES_LIMIT = 12,      /* "GMRES iteration limit reached" linear.cpp:155 */
  EG_ERR_LINEAR_RESIDUAL = 13,  /* "True inverse-mass weighted linear residual too large" linear.cpp:246 */
  EG_ERR_RECOVERED = 14,        /* "Recovered DG residual criterion failed after Schur refinement" stepper.cpp:180 */
  EG_ERR_DG_LINEAR = 15,        /* "DG Newton linear residual too large" stepper.cpp:183 */
  EG_ERR_LINE_SEARCH = 16,      /* "Newton line search failed" stepper.cpp:217 */
  EG_ERR_OUT_OF_MEMORY = 17,    /* device allocation failed */
  EG_ERR_STEP_INTERVAL = 18,    /* "Step leaves the smooth simple-wave interval ..." stepper.cpp:94-95 */
  EG_ERR_NEWTON_CONVERGE = 19,  /* "Newton failed to converge" stepper.cpp:241 */
  EG_ERR_DIRK_INADMISSIBLE = 20,/* "SSP-DIRK3 step produced an inadmissible state" stepper.cpp:251 */
  EG_ERR_INITIAL = 21,          /* "Initial projection not positive; refine mesh" stepper.cpp:32 */
  EG_ERR_UPDATE_EQUATION = 22,  /* "Independent recovered DG equation check failed" stepper.cpp:190 */
  EG_ERR_UPDATE_EQUIVALENCE = 23, /* "DG/HDG one-update equivalence failed" stepper.cpp:197 */
  EG_ERR_WAIT_LIMIT = 24,       /* a bounded device-side wait gave up: a dependency-driven block
                                   ILU(0) factor or sweep, or a bulk copy of the DG block-Jacobi
                                   record apply (no counterpart in the reference, whose factor and
                                   sweeps are serial); the context stays usable */
  EG_ERR_CONTEXT_LOST = 25,     /* after a wait gave up, a bulk copy of the aborted sweep did not
                                   land within its own bound either: the context's device memory
                                   can no longer be trusted, every later call on it returns this
                                   status, and only eg_destroy is valid (no reference counterpart) */
  EG_ERR_COUNT = 26
};

enum eg_form { EG_FORM_DG = 0, EG_FORM_HDG = 1 };
enum eg_precond { EG_PC_BLOCK_JACOBI = 0, EG_PC_BLOCK_ILU0 = 1 };
/* Options::assembly (src/options.cpp:51-53, 130-146):
 *  PARTIAL  matrix-free operators (DG: PartialDGOperator; HDG: the Schur action from C and X);
 *  ELEMENT  element-assembled operators applied matrix-free (DG: the cell and face-coupling
 *           blocks of the Jacobian; HDG: the per-cell Schur entries C X, src/condensation.cpp:143-146);
 *  FULL     GMRES on the assembled block-sparse matrix (ElementOperator::Assemble,
 *           src/operators.cpp:180-238), the final residual from the element operator
 *           (src/linear.cpp:242-246). */
enum eg_assembly { EG_ASSEMBLY_PARTIAL = 0, EG_ASSEMBLY_FULL = 1, EG_ASSEMBLY_ELEMENT = 2 };
enum eg_precision {
  EG_PRECISION_FP64 = 0,  /* everything FP64 (parity path) */
  EG_PRECISION_MIXED = 1  /* FP32 preconditioner + FP32 inner Schur GMRES in FP64 refinement */
};

/* Named device vectors of a context (eg_upload / eg_download). */
enum eg_slot {
  EG_SLOT_U = 0,       /* Newton state (nu) */
  EG_SLOT_OLD = 1,     /* stage base / old state (nu) */
  EG_SLOT_R = 2,       /* stored residual M^{-1} r_w + u - old (nu) */
  EG_SLOT_DU = 3,      /* last Newton increment (nu) */
  EG_SLOT_RHS = 4,     /* condensed Schur right-hand side (nl) */
  EG_SLOT_LAMBDA = 5,  /* last Schur solution (nl) */
  EG_SLOT_D = 6,       /* HDG trace diagonal D (nl) */
  EG_SLOT_X = 7,       /* HDG responses X, n blocks of m x 4t column-major */
  EG_SLOT_Y = 8,       /* HDG particular responses y (nu) */
  EG_SLOT_PC_BLOCKS = 9, /* preconditioner blocks, column-major (count: eg_pc_size).
                          block-jacobi: DG n*m*m, HDG nf*t*t; after eg_pc_factor(ctx, 1) HDG
                          and DG with k <= 5 hold explicit inverses (DG column-major; for
                          k = 3..5 the device keeps a Gauss-Jordan record and the
                          download expands it into the inverses it applies), DG
                          with k >= 6 packed pivoted LU.
                          block-ilu0: the BSR blocks of the ILU in FixedBlockILU order (rows
                          ascending, block columns ascending); after eg_pc_factor(ctx, 1) the
                          strictly lower blocks hold L, the others U (diagonal unfactored). */
  EG_SLOT_HLL_A = 10,  /* frozen left HLL bound per face point (nf*q) */
  EG_SLOT_HLL_B = 11,  /* frozen right HLL bound per face point (nf*q) */
  EG_SLOT_COUNT = 12
};

/* Problem description: geometry and the reference's host-computed tables
 * (src/problem.cpp:32-222). Fixed-size arrays hold q <= EG_MAX_Q. */
typedef struct eg_desc {
  int nx, ny, k;
  double gamma;        /* EulerGas gamma (src/main.cpp:8 uses 3) */
  double safety;       /* HLL safety factor (Options::safety) */
  double alpha;        /* wave angle in radians */
  double lx, ly, hx, hy, area;
  double w[EG_MAX_P];        /* volume GL weights, native node order */
  double ew[EG_MAX_Q];       /* edge GL weights */
  double ex[EG_MAX_Q];       /* edge GL points in [0,1] */
  double inv_mass[EG_MAX_P]; /* diagonal of Problem::inv_mass */
  double mass[EG_MAX_P];     /* diagonal of Problem::mass */
  double tensor_dx[EG_MAX_P]; /* Problem::tensor_dx(a,i) at [a*q+i] */
  double tensor_dy[EG_MAX_P]; /* Problem::tensor_dy(a,j) at [a*q+j] */
  /* fv[s](j, node) along the normal line through face point j of side s:
   * [(s*q + j)*q + l], node = j*q+l for s<2 and l*q+j for s>=2. */
  double face_basis[4 * EG_MAX_Q * EG_MAX_Q];
  int tensor_node[EG_MAX_P]; /* lexicographic -> native; must be the identity */
} eg_desc;

/* Solver options (the numerical subset of euler::Options, include/euler.hpp:46-57). */
/* Linear solver of the Newton system: restarted GMRES, or the dense direct
 * LU of the full assembly (--solver dense; --solver direct needs MKL PARDISO,
 * which neither the reference's portable build nor this library has). */
enum eg_solver { EG_SOLVER_GMRES = 0, EG_SOLVER_DENSE = 1 };

typedef struct eg_opts {
  int form;        /* eg_form */
  int precond;     /* eg_precond */
  int assembly;    /* eg_assembly */
  int precision;   /* eg_precision */
  int restart;     /* GMRES restart (default 20) */
  int max_krylov;  /* GMRES iteration limit (default 1500) */
  double linear_tol; /* default 1e-12 */
  int check_update;  /* HDG: independent DG solve of every update (stepper.cpp:184-201) */
  int solver;        /* eg_solver (Options::solver, src/options.cpp:56-57, 111-112):
                        EG_SOLVER_DENSE needs EG_ASSEMBLY_FULL, FP64 and at most 5000
                        unknowns in the solved system (src/linear.cpp:46-47) */
} eg_opts;

/* Per-update statistics: the numeric columns of _iterations.csv
 * (src/stepper.cpp:229-239). Times are seconds. */
typedef struct eg_update_stats {
  double residual_norm;  /* CellNorm(residual) before the update */
  double damping;
  int krylov_iterations;
  int attempts;          /* Schur refinement attempts (HDG) */
  double linear_relative_residual;
  double dg_linear_relative_residual;
  double residual_s, validation_s, jacobian_s, condensation_s, assembly_s, setup_s,
      solve_s, recovery_s, line_search_s, iteration_s;
  double device_ms;      /* CUDA-event time of the whole update on the context stream */
  double update_check;   /* --check-update relative difference, -1 when not run */
} eg_update_stats;

/* Linear-solve statistics (LinearResult, include/euler.hpp:232-236). */
typedef struct eg_linear_stats {
  int count;
  double residual;  /* relative weighted residual */
  double rhs_norm;
} eg_linear_stats;

typedef struct eg_ctx eg_ctx;

/* ---------------------------------------------------------------- setup */
/* Fill a descriptor for the rotated simple-wave problem on an nx x ny periodic
 * Qk mesh, computing the Gauss-Legendre tables on the host exactly as the
 * reference Problem constructor does (src/problem.cpp:32-222). */
int eg_desc_simple_wave(eg_desc *d, int nx, int ny, int k, double alpha_deg, double gamma,
                        double safety);
void eg_opts_default(eg_opts *o);
/* Select the CUDA device for contexts created later on the calling thread
 * (the library links its own CUDA runtime, so callers that chose a device
 * through another runtime must select it here as well). */
int eg_set_device(int device);

/* Replaces: Problem construction + PrepareHybrid + LinearSolver construction
 * (src/problem.cpp:32, src/condensation.cpp:47, src/linear.cpp:159). */
int eg_create(const eg_desc *d, const eg_opts *o, eg_ctx **out);
void eg_destroy(eg_ctx *ctx);
/* Message of the last failure on ctx; with ctx == NULL, of the last failed
 * eg_create on the calling thread. */
const char *eg_last_error(const eg_ctx *ctx);
const char *eg_status_string(int status);
/* cudaStream_t of the context, as void*. */
void *eg_stream(eg_ctx *ctx);
/* Re-describe a context for another problem of the same nx, ny and k (angle,
 * box, gas, tables): the device buffers are kept, the state must be set anew.
 * No counterpart in the reference (one Problem per run). */
int eg_set_desc(eg_ctx *ctx, const eg_desc *d);
/* Change solver options between updates (form, preconditioner, tolerance).
 * The assembly mode is fixed when the context is created (it decides how many
 * Schur panels the condensation keeps); a different one is EG_ERR_INVALID. */
int eg_set_opts(eg_ctx *ctx, const eg_opts *o);
/* Sizes: n, p, m, t, nf, nu, nl. */
int eg_sizes(const eg_ctx *ctx, int out[7]);
/* Device bytes held by the context. */
long long eg_device_bytes(const eg_ctx *ctx);

/* --------------------------------------------------------- state access */
int eg_upload(eg_ctx *ctx, int slot, const double *src);
int eg_download(eg_ctx *ctx, int slot, double *dst);
/* Replaces: Problem::Initial (src/problem.cpp:329), L2 projection of the exact
 * wave at t=0 into EG_SLOT_U, computed on the device (order max(24, 2k+8)
 * Gauss-Legendre rule, EulerGas::exact src/physics.cpp:64). */
int eg_initial(eg_ctx *ctx);

/* ---------------------------------------------------- operators (parity) */
/* Replaces: Problem::Freeze (src/problem.cpp:350) at EG_SLOT_U, including
 * old = u and dt = stage_dt; writes WaveRate (problem.cpp:377) if non-null. */
int eg_freeze(eg_ctx *ctx, double stage_dt, int check_admissible, double *wave_rate);
/* Sets Problem::dt (used after Freeze by the time loop, stepper.cpp:109). */
int eg_set_dt(eg_ctx *ctx, double dt);
/* Replaces: Problem::Residual (src/problem.cpp:445): EG_SLOT_R <- r(EG_SLOT_U). */
int eg_residual(eg_ctx *ctx);
/* Replaces: Problem::CellNorm (src/problem.cpp:385) of a body slot. */
int eg_cell_norm(eg_ctx *ctx, int slot, double *out);
/* Replaces: Problem::Admissible (src/problem.cpp:259) of a body slot. */
int eg_admissible(eg_ctx *ctx, int slot, int *ok);
/* Replaces: PartialDGOperator::Refresh + Mult (src/partial.cpp:31-135):
 * y = J(EG_SLOT_U) x, nu-vectors. */
int eg_dg_apply(eg_ctx *ctx, const double *x, double *y);
/* Replaces: Problem::StreamCondense (src/condensation.cpp:131) at EG_SLOT_U
 * with residual EG_SLOT_R: fills X, y, D and the Schur right-hand side. */
int eg_condense(eg_ctx *ctx);
/* Replaces: ElementOperator::Mult with borrowed factors (src/operators.cpp:147):
 * Schur action y = D v - sum_e C_e X_e v_e, nl-vectors. */
int eg_schur_apply(eg_ctx *ctx, const double *v, double *y);
/* Replaces: Problem::Recover (src/condensation.cpp:154): du = -X lam - y. */
int eg_recover(eg_ctx *ctx, const double *lam, double *du);
/* Replaces: the preconditioner refresh in LinearSolver::Solve
 * (src/linear.cpp:186-203): DiagonalBlocks+LU or FillBlocks+ILU factor for the
 * current form. factor=0 stops after building (for EG_SLOT_PC_BLOCKS parity). */
int eg_pc_factor(eg_ctx *ctx, int factor);
/* Number of doubles in EG_SLOT_PC_BLOCKS for the current form and
 * preconditioner (0 before the first eg_pc_factor with block-ilu0). */
int eg_pc_size(const eg_ctx *ctx, long long *count);
/* Replaces: LinearSolver::Impl::Precondition (src/linear.cpp:66) with block
 * Jacobi, FixedBlockILU::Mult (src/block_ilu.cpp:88) with block-ilu0. */
int eg_pc_apply(eg_ctx *ctx, const double *b, double *x);
/* Replaces: LinearSolver::Solve (src/linear.cpp:167) for the current form:
 * weighted right-preconditioned restarted CGS2 GMRES. x is in/out (used as
 * the initial guess when refresh == 0); eq_residual (may be null) receives
 * op*x - rhs. */
int eg_linear_solve(eg_ctx *ctx, const double *rhs, double *x, double *eq_residual,
                    int refresh, double linear_tol, eg_linear_stats *st);

/* ------------------------------------------------------- Newton / stages */
/* Stage setup (src/stepper.cpp:99-110): dt = stage_dt and EG_SLOT_OLD
 * already uploaded or set; marks the stored residual stale. */
int eg_stage_begin(eg_ctx *ctx, double stage_dt);
/* Newton residual (stepper.cpp:118-121): recomputes EG_SLOT_R unless the last
 * accepted line-search residual is still valid; returns CellNorm(r). */
int eg_newton_residual(eg_ctx *ctx, double *residual_norm);
/* One accepted damped Newton update (src/stepper.cpp:129-228), DG or HDG per
 * the context's form: Jacobian / condensation, PC, GMRES, recovery and the
 * recovered-residual refinement loop, validation and line search, all on the
 * device. old_norm = CellNorm(stage base). */
int eg_newton_update(eg_ctx *ctx, double residual_norm, double old_norm, eg_update_stats *st);

/* --------------------------------------------------------- diagnostics */
/* Replaces: Problem::Integral (src/problem.cpp:727) of EG_SLOT_U (device). */
int eg_integral(eg_ctx *ctx, double out[4]);
/* Replaces: Problem::Errors (src/problem.cpp:704) of EG_SLOT_U at time t
 * (device; EG_ERR_STEP_INTERVAL for t outside the exact wave's interval). */
int eg_errors(eg_ctx *ctx, double time, double out[4]);
/* Replaces: Problem::Differences (src/problem.cpp:739) of EG_SLOT_U and v, a
 * host or device body vector (device computation). */
int eg_state_differences(eg_ctx *ctx, const double *v, double out[4]);
/* Replaces: Problem::Differences (src/problem.cpp:739): L2 norms of u - v per
 * component for two host body vectors of the described problem, on the host
 * (no context needed; eg_state_differences is the device form). */
int eg_differences(const eg_desc *d, const double *u, const double *v, double out[4]);
/* Replaces: Problem::Save (src/problem.cpp:762-790) for a host body vector u:
 * writes prefix.mesh (MFEM mesh v1.0 text of the Cartesian quadrilateral
 * mesh), prefix_{rho,rhou,rhov,energy}.gf (one L2 Gauss-Legendre grid
 * function per component) and prefix_coefficients.csv. Host only; no context
 * needed. EG_ERR_INVALID (message in eg_last_error(NULL)) when a file cannot
 * be opened. */
int eg_save_solution(const eg_desc *d, const double *u, const char *prefix);

/* ------------------------------------------------------------ time loop */
/* Run options: the time-loop subset of euler::Options. */
typedef struct eg_run_opts {
  int integrator;     /* 0 = ssp-dirk3, 1 = be */
  int steps;          /* > 0: fixed step count; else run to T */
  int newton_steps;   /* > 0: fixed updates per stage; else converge */
  int max_newton;
  double dt, cfl, end, tol;
  int timing_only, save_solution;
  const char *prefix; /* output prefix, e.g. "<output>_dg" */
  const char *form_name; /* "dg" or "hdg" for CSV rows */
  /* echoed into _summary.csv */
  const char *assembly_name, *solver_name, *precond_name, *ilu_ordering_name;
  int check_update;
} eg_run_opts;

typedef struct eg_run_result {
  double errors[4];
  double seconds, drift, newton_seconds, final_time, mean_newton_s;
  double newton_device_ms; /* sum of per-update CUDA-event times */
  int updates, time_steps;
} eg_run_result;

/* Replaces: euler::Run (src/stepper.cpp:28-292), writing the same
 * _iterations.csv / _summary.csv columns. The final state stays in EG_SLOT_U. */
int eg_run(eg_ctx *ctx, const eg_run_opts *ro, eg_run_result *res);

/* Incremental time loop for benchmarks: advances the SSP-DIRK3/BE schedule by
 * exactly one accepted Newton update per call (stage and step transitions,
 * Freeze and DIRK combination are performed between updates, outside the
 * update's timed boundary). */
typedef struct eg_stepper eg_stepper;
int eg_stepper_create(eg_ctx *ctx, const eg_run_opts *ro, eg_stepper **out);
int eg_stepper_next(eg_stepper *s, eg_update_stats *st);
void eg_stepper_destroy(eg_stepper *s);
/* After eg_stepper_next returned -1: final time, step count, L2 errors against
 * the exact wave (Problem::Errors, src/problem.cpp:704) and the conservation
 * drift of the final state (src/stepper.cpp:255-258). The update counters of
 * res are left zero (the caller counts its eg_stepper_next calls). */
int eg_stepper_finish(eg_stepper *s, eg_run_result *res);

/* ------------------------------------- many instances: batch and serving */
/* Neither has a counterpart in the reference, whose driver runs one problem
 * per process. Every instance is an eg_ctx with its own CUDA stream; host
 * worker threads advance the instances through the calls above, so the
 * Newton updates of different instances overlap on the GPU. Each instance's
 * kernels and reductions are the single-instance ones, so every result is
 * bitwise the one the instance gives when run alone. */

/* A fixed set of instances run to completion together (uneven nx, ny, k). */
typedef struct eg_batch eg_batch;
typedef struct eg_batch_stats {
  double seconds;          /* wall time of eg_batch_run */
  long long updates;       /* accepted Newton updates over all instances */
  int failed;              /* instances whose run returned an error */
} eg_batch_stats;
/* count instances: descs[i] with opts[i], on `device`. */
int eg_batch_create(int count, const eg_desc *descs, const eg_opts *opts, int device, eg_batch **out);
/* Runs every instance through the schedule ro on `threads` host workers. */
int eg_batch_run(eg_batch *b, const eg_run_opts *ro, int threads, eg_batch_stats *st);
/* Per-instance outcome: status, updates and the final errors/drift. */
int eg_batch_result(const eg_batch *b, int i, int *status, eg_run_result *res);
/* The instance's context (its final state is EG_SLOT_U). */
eg_ctx *eg_batch_context(eg_batch *b, int i);
void eg_batch_destroy(eg_batch *b);

/* A request loop: time-advance requests are submitted while others run;
 * a request is admitted when a worker is free and its device memory fits the
 * budget beside the requests already resident (first come, first served). */
typedef struct eg_server eg_server;
typedef struct eg_server_opts {
  int device;
  int workers;              /* concurrent requests on the GPU */
  long long budget_bytes;   /* device memory budget of resident requests */
  int keep_contexts;        /* reuse finished contexts of the same shape */
  int keep_states;          /* copy each final state to host memory (eg_server_state) */
} eg_server_opts;
typedef struct eg_request {
  int nx, ny, k;
  double alpha_deg;
  int steps, newton_steps;  /* SSP-DIRK3 steps; updates per stage (<= 0: converge) */
  double cfl;
  int form, precond, precision;
} eg_request;
typedef struct eg_request_result {
  int status;               /* EG_OK or the failing call's status */
  int updates;
  double submit_s, start_s, finish_s;   /* server clock, seconds */
  double final_time, errors[4], drift;
  long long bytes;          /* device bytes charged against the budget */
} eg_request_result;
typedef struct eg_server_stats {
  long long completed, failed;
  long long peak_bytes;     /* largest sum of resident request bytes */
  int peak_running;         /* largest number of requests on the GPU at once */
} eg_server_stats;
int eg_server_create(const eg_server_opts *o, eg_server **out);
/* Queues a request; *id identifies it. Never blocks on the GPU. */
int eg_server_submit(eg_server *s, const eg_request *r, long long *id);
/* EG_OK when the request has finished (res filled), -1 while pending. */
int eg_server_poll(eg_server *s, long long id, eg_request_result *res);
/* Copies the final state (nx*ny*4(k+1)^2 doubles) of a finished request. */
int eg_server_state(eg_server *s, long long id, double *u);
/* Blocks until every submitted request has finished. */
int eg_server_drain(eg_server *s, eg_server_stats *st);
/* Seconds on the server clock (the time base of eg_request_result). */
double eg_server_clock(const eg_server *s);
void eg_server_destroy(eg_server *s);

/* ------------------------------------------------- allocation-free entry */
/* CellNorm of a body vector without any device allocation. This entry point
 * has no counterpart in the reference.
 *
 * It exists for callers that may not allocate device memory from library
 * code: applications whose device memory is owned by their own allocator or
 * memory pool (every buffer handed out and accounted for by that pool), and
 * deployments that fix the device-memory footprint in advance. Such a caller
 * cannot create an eg_ctx, because a context allocates its buffers.
 *
 * r must point to n*m doubles of device-accessible memory laid out as the
 * reference's body vectors, on the current device (host pointers and memory
 * of another device are rejected with EG_ERR_INVALID, as is a descriptor that
 * eg_create would refuse: non-lexicographic nodes or a non-positive area);
 * *out receives sqrt(sum_i area * mass_i * r_i^2), the same value eg_cell_norm
 * returns for the same vector. stream may be NULL (the default stream).
 *
 * The call is synchronous: it copies the metric table from the host, runs the
 * reduction and waits on the stream for the result, so it must not be called
 * while its stream is being captured into a CUDA graph.
 *
 * Scratch: a fixed 4 KB static device array inside the library (partial sums,
 * completion counter, metric table), held by every GPU that loads the library
 * until the process exits. Degrees k > 8 exceed its metric table and are
 * rejected with EG_ERR_INVALID. The first call on each device looks up the
 * array's device address with that device current. All calls on a device
 * share the array, so calls that overlap on the GPU (concurrent streams or
 * threads) race and must be serialised by the caller. */
int eg_cell_norm_noalloc(const eg_desc *d, const double *r, void *stream, double *out);

/* ------------------------------------------------------------ profiling */
/* Kernel classes timed with CUDA events on the context stream when
 * profiling is on (eg_profile_enable). */
enum eg_kernel_class {
  EG_K_RESIDUAL = 0, EG_K_DG_APPLY = 1, EG_K_DG_JACOBI = 2, EG_K_CONDENSE = 3,
  EG_K_SCHUR_APPLY = 4, EG_K_RECOVER = 5, EG_K_RECOVERED_RESIDUAL = 6, EG_K_SCHUR_JACOBI = 7,
  EG_K_PC_APPLY = 8, EG_K_KRYLOV = 9, EG_K_FREEZE = 10, EG_K_ADMISSIBLE = 11, EG_K_VECTOR = 12,
  EG_K_COUNT = 13
};
int eg_profile_enable(eg_ctx *ctx, int on);
int eg_profile_reset(eg_ctx *ctx);
/* Accumulated device milliseconds and launch count of one kernel class since
 * the last reset (synchronises the context stream). */
int eg_profile_query(eg_ctx *ctx, int kernel_class, double *ms, long long *launches);
/* Total kernels launched on the context since creation. */
long long eg_launch_count(const eg_ctx *ctx);

/* y[i] = the condensation's pivot reciprocal of x[i] (host arrays of n
 * values), for tests that bound it against IEEE division (no reference
 * counterpart: the reference divides by each pivot). */
int eg_check_pivot_reciprocal(const double *x, double *y, long long n);

/* Test setting of the block ILU(0) device waits (no reference counterpart:
 * the reference's factor and sweeps are serial). limit_ns bounds every wait
 * of the factor and the sweeps (0 restores the default, 250 ms); starve != 0
 * makes every wait on another CTA unreachable, so that the next factor or
 * apply runs out its bound, returns EG_ERR_WAIT_LIMIT and leaves the context
 * usable. Applies to both forms' plans, including ones built later. */
int eg_set_ilu_wait(eg_ctx *ctx, unsigned long long limit_ns, int starve);

#ifdef __cplusplus
}
#endif
#endif /* EULER2D_CUDA_H */
