/*
 * ewg.h -- C ABI of the B200 element-centred finite-volume (ECFV) linearizer and the
 * BiCGStab / block-ILU0 / block-Jacobi solver for the immiscible two-phase model.
 *
 * The entry points replace, one for one, the pieces of eWoms' hot path that a Problem/Model
 * reaches through the property system:
 *
 *   FvBaseLinearizer            discretizations/common/fvbaselinearizer.hh
 *   FvBaseAdLocalLinearizer     discretizations/common/fvbaseadlocallinearizer.hh
 *   ParallelBiCGStabSolverBackend / ParallelBaseBackend
 *                               linear/parallelbicgstabbackend.hh, linear/parallelbasebackend.hh
 *   BiCGStabSolver + CombinedCriterion
 *                               linear/bicgstabsolver.hh, linear/combinedcriterion.hh
 *   NewtonMethod::apply         nonlinear/newtonmethod.hh
 *
 * Conventions
 *   - Plain C types only. Host pointers are borrowed for the duration of a call and copied.
 *   - Cell vectors on the host are in the reference's natural (lexicographic, x fastest) order,
 *     one 2-block per cell: {p_w, S_w} for primary variables, {conti_w, conti_n} for residuals
 *     (pressure0Idx = 0, saturation0Idx = 1, conti0EqIdx = 0; models/immiscible/immiscibleindices.hh).
 *   - Jacobian blocks are 2x2, row-major [eqIdx][pvIdx]; J[row j][col i] = dR_j / dx_i, the layout
 *     FvBaseLinearizer::linearizeElement_ scatters (fvbaselinearizer.hh:496-508).
 *   - Every function returns an ewg_status. Non-zero means failure; ewg_last_error() explains.
 *     A caller mapping non-zero to Ewoms::NumericalIssue keeps the reference's time-step halving
 *     (fvbaseproblem.hh:507-550) unchanged.
 *   - One context owns all device buffers and one CUDA stream. Calls on one context are not
 *     reentrant. There is no CPU fallback: without a usable CUDA device ewg_create fails with
 *     EWG_ERR_NO_DEVICE.
 */
#ifndef EWG_H
#define EWG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EWG_ABI_VERSION 1

typedef enum ewg_status {
    EWG_OK = 0,
    EWG_ERR_INVALID = 1,        /* bad argument or unsupported configuration */
    EWG_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    EWG_ERR_NONFINITE = 3,      /* NaN/Inf in residual, gradient or Newton update */
    EWG_ERR_BREAKDOWN = 4,      /* BiCGStab breakdown / stagnation (bicgstabsolver.hh:196,228,284) */
    EWG_ERR_NOT_CONVERGED = 5,  /* linear or Newton iteration did not converge */
    EWG_ERR_TIMEOUT = 6,        /* a bounded device wait gave up */
    EWG_ERR_NO_DEVICE = 7,      /* no CUDA device, or the device is not sm_100 */
    EWG_ERR_MAX_ERROR = 8       /* Newton error above NewtonMaxError (newtonmethod.hh:681-684) */
} ewg_status;

/* Structured grid (StructuredGridVanguard, io/structuredgridvanguard.hh:136-175). The domain is
 * [0,lx] x [0,ly] (x [0,lz]) with uniform cells; gravity acts along -y in 2D and 3D
 * (multiphasebaseproblem.hh:393-398, lensproblem.hh:284-287). nx must be even: the device stores
 * cells in red-black split order. */
typedef struct ewg_grid {
    int32_t dim;                /* 2 or 3 */
    int32_t nx, ny, nz;         /* nz is ignored (treated as 1) for dim == 2 */
    double lx, ly, lz;          /* extents [m]; lz ignored for dim == 2 */
    int32_t k_origin;           /* global index of the first z-plane: 0 for a whole grid; for one
                                   z-slab of a decomposed 3D grid, its first plane, so that plane k
                                   sits at z = (k_origin + k + 1/2) lz / nz and the lens and inlet
                                   boxes keep their global coordinates (cell-centred contexts only) */
} ewg_grid;

typedef enum ewg_law_kind {
    EWG_LAW_VAN_GENUCHTEN = 0,  /* EffToAbsLaw<RegularizedVanGenuchten> (lensproblem.hh:107-126) */
    EWG_LAW_BROOKS_COREY = 1    /* EffToAbsLaw<RegularizedBrooksCorey> (tutorial/tutorial1problem.hh:86-104) */
} ewg_law_kind;

/* Material-law parameters of one region (lensproblem.hh:266-279). */
typedef struct ewg_material {
    int32_t law;                /* ewg_law_kind */
    double swr, snr;            /* residual saturations of the wetting / non-wetting phase */
    double vg_alpha, vg_n;      /* van Genuchten alpha [1/Pa] and n */
    double bc_entry_pressure;   /* Brooks-Corey entry pressure [Pa] */
    double bc_lambda;           /* Brooks-Corey shape parameter */
} ewg_material;

/* Boundary-face kinds of the lens problem (LensProblem::boundary, lensproblem.hh:464-533). */
typedef struct ewg_problem {
    double lens_lo[3], lens_hi[3];  /* lens box (isInLens_, lensproblem.hh:596-604) */
    double eps;                     /* geometric tolerance, 3e-6 in the reference */
    double porosity;                /* 0.4 */
    double temperature;             /* 293.15 K; carried for completeness (liquids are constant) */
    double rho_w, mu_w;             /* wetting liquid density [kg/m^3], viscosity [Pa s] */
    double rho_n, mu_n;             /* non-wetting liquid */
    double gravity;                 /* magnitude [m/s^2]; the vector is (0,-g[,0]) */
    double p_ref;                   /* pressure at the top (y = ly), 1e5 Pa */
    double left_pressure_scale;     /* hydrostatic factor on the left boundary: 1 + 1.5/H in the
                                       reference (lensproblem.hh:481-488), 1 for plain Dirichlet */
    double inlet_x_lo, inlet_x_hi;  /* inlet on the top face for inlet_x_lo < x < inlet_x_hi */
    double inlet_z_lo, inlet_z_hi;  /* 3D only: and inlet_z_lo < z < inlet_z_hi */
    double inlet_rate;              /* mass rate on the non-wetting equation [kg/(m^2 s)], -0.04 */
    ewg_material outer;             /* material outside the lens */
    ewg_material lens;              /* material inside the lens */
} ewg_problem;

/* LocalLinearizerSplice: how the local Jacobian of an element is formed. */
typedef enum ewg_local_linearizer {
    EWG_LOCAL_LINEARIZER_AD = 0,  /* AutoDiffLocalLinearizer (fvbaseadlocallinearizer.hh:178-297), default */
    EWG_LOCAL_LINEARIZER_FD = 1   /* FiniteDifferenceLocalLinearizer (fvbasefdlocallinearizer.hh:221-453) */
} ewg_local_linearizer;

typedef enum ewg_precond_kind {
    EWG_PRECOND_ILU0 = 0,       /* block ILU(0) in the row order of ewg_solve_opts.ilu_ordering */
    EWG_PRECOND_JACOBI = 1      /* block Jacobi, one sweep with relaxation */
} ewg_precond_kind;

typedef enum ewg_precision {
    EWG_PRECISION_FP64 = 0,     /* Jacobian, preconditioner and BiCGStab in FP64 */
    EWG_PRECISION_MIXED = 1     /* FP32 Jacobian copy, FP32 preconditioner and BiCGStab inside an
                                   FP64 defect-correction loop */
} ewg_precision;

/* Row order of the block ILU(0) preconditioner. The reference factorizes in the grid's natural
 * (lexicographic) order, whose triangular sweeps are sequential; the device uses parallel orders:
 *   REDBLACK  two colours by (i + j + k) parity: red rows, then black rows (2D and any even nx);
 *   BOX8      2x2x2 boxes in eight colours by bit 1 of (i, j, k), natural order inside a box
 *             (3D grids with nx, ny, nz multiples of 4): about a third fewer BiCGStab iterations
 *             than REDBLACK on the lens problem;
 *   AUTO      BOX8 where the grid allows it, else REDBLACK.
 * ewg_solve, ewg_apply_preconditioner and ewg_device_precondition take it from the options. */
typedef enum {
    EWG_ILU_ORDER_AUTO = 0,
    EWG_ILU_ORDER_REDBLACK = 1,
    EWG_ILU_ORDER_BOX8 = 2
} ewg_ilu_ordering;

/* Linear-solver parameters; names follow the reference's runtime parameters. */
typedef struct ewg_solve_opts {
    int32_t precond;                  /* ewg_precond_kind */
    int32_t precision;                /* ewg_precision */
    double linear_solver_tolerance;   /* LinearSolverTolerance (relative max-norm reduction) */
    double linear_solver_abs_tolerance; /* LinearSolverAbsTolerance (max-norm) */
    double linear_solver_max_error;   /* LinearSolverMaxError, 1e7 */
    int32_t linear_solver_max_iterations; /* LinearSolverMaxIterations, 1000 */
    double preconditioner_relaxation; /* PreconditionerRelaxation, 1.0 */
    /* mixed precision only: FP64 defect-correction loop */
    double defect_tolerance;          /* stop when max|b - A x| <= this (FP64); <= 0: same as abs tol */
    double inner_tolerance;           /* relative reduction asked of each FP32 inner solve */
    int32_t max_defect_iterations;
    int32_t check_interval;           /* BiCGStab iterations between host status reads; 0 = auto */
    int32_t restart_on_breakdown;     /* 1: when |r0hat . r| <= 1e-12 |r0hat| |r| at the top of an
                                         iteration, restart with r0hat = r (x kept). 0: exactly the
                                         reference, which then breaks down (EWG_ERR_BREAKDOWN) */
    int32_t verify_true_residual;     /* 1: on convergence recompute b - A x; if it misses the
                                         criterion by more than 10x, continue from x with the true
                                         residual (at most 3 replacements). 0: exactly the reference */
    int32_t ilu_ordering;             /* ewg_ilu_ordering: the row order block ILU(0) factorizes in */
} ewg_solve_opts;

typedef struct ewg_solve_report {
    int32_t converged;
    int32_t restarts;                 /* shadow-residual restarts and residual replacements */
    int32_t iterations;               /* BiCGStab iterations (sum over defect-correction passes) */
    int32_t outer_iterations;         /* defect-correction passes (1 for FP64) */
    int32_t status;                   /* ewg_status of the solve */
    double initial_residual;          /* max|b| */
    double final_residual;            /* max-norm of the last checked residual */
    double seconds;                   /* device time of the solve */
} ewg_solve_report;

typedef struct ewg_lin_report {
    double error;                     /* max over cells and equations of |r| (newtonmethod.hh:659-674) */
    int32_t nonfinite;                /* 1 if any residual entry is NaN/Inf */
    double seconds;                   /* device time of the linearization */
} ewg_lin_report;

typedef struct ewg_newton_opts {
    double newton_tolerance;          /* NewtonTolerance, 1e-8 */
    double newton_max_error;          /* NewtonMaxError, 1e100 */
    int32_t newton_max_iterations;    /* NewtonMaxIterations, 18 */
    int32_t newton_target_iterations; /* NewtonTargetIterations, 10 */
    int32_t verbose;
} ewg_newton_opts;

typedef struct ewg_newton_report {
    int32_t converged;
    int32_t iterations;               /* Newton iterations (numIterations_) */
    int32_t linear_iterations;        /* BiCGStab iterations summed over the Newton iterations */
    int32_t status;
    double error;                     /* last Newton error */
    double t_linearize, t_solve, t_update;  /* device seconds per phase (newtonmethod.hh:488-500) */
} ewg_newton_report;

typedef struct ewg_ctx ewg_ctx;

/* ---- context ------------------------------------------------------------------------ */

/* Build the device problem: geometry, per-cell permeability (natural order, N doubles, isotropic
 * K [m^2]; NULL = lens/outer constants are not given here, so perm is required) and the
 * precomputed 7-band (3D) / 5-band (2D) block pattern of the Jacobian. Replaces
 * FvBaseLinearizer::init + createMatrix_ (fvbaselinearizer.hh:284-340). */
ewg_status ewg_create(const ewg_grid* grid, const ewg_problem* problem, const double* perm,
                      ewg_ctx** out);
void ewg_destroy(ewg_ctx* ctx);
const char* ewg_last_error(const ewg_ctx* ctx);
/* Last error of a failed ewg_create (no context exists yet). */
const char* ewg_create_error(void);
int64_t ewg_num_cells(const ewg_ctx* ctx);
/* Number of 2x2 blocks of the reference's BCRS pattern: N + 2 * interior faces. */
int64_t ewg_num_blocks(const ewg_ctx* ctx);
int32_t ewg_abi_version(void);

/* ---- solution history (FvBaseDiscretization::solution(timeIdx)) -------------------- */

/* time_idx 0: current Newton iterate; time_idx 1: solution of the previous time level. x is
 * N x {p_w, S_w}. Setting time_idx 1 also recomputes the old-time storage term from it
 * (fvbaselocalresidual.hh:538-575 with the storage cache). */
ewg_status ewg_set_solution(ewg_ctx* ctx, int32_t time_idx, const double* x);
ewg_status ewg_get_solution(ewg_ctx* ctx, int32_t time_idx, double* x);
/* Hydrostatic initial condition of LensProblem::initial (lensproblem.hh:545-578) into both levels. */
ewg_status ewg_apply_initial_solution(ewg_ctx* ctx);
/* advanceTimeLevel (fvbasediscretization.hh:1396-1407): solution(1) = solution(0). */
ewg_status ewg_advance_time_level(ewg_ctx* ctx);
/* updateFailed (fvbasediscretization.hh:1370-1387): solution(0) = solution(1). */
ewg_status ewg_restore_time_level(ewg_ctx* ctx);

/* ---- FvBaseLinearizer ---------------------------------------------------------------- */

/* Select the local linearizer (SET_TAG_PROP(..., LocalLinearizerSplice, ...)). For
 * EWG_LOCAL_LINEARIZER_FD, numeric_difference_method is NumericDifferenceMethod: -1 backward,
 * 0 central, +1 forward differences (the reference's default); the deflection is
 * BaseEpsilon / primaryVarWeight with the pressure weight 10 / p_ref (immisciblemodel.hh:298-310). */
ewg_status ewg_set_local_linearizer(ewg_ctx* ctx, int32_t kind, int32_t numeric_difference_method);
/* FvBaseDiscretization::updateBegin (ImmiscibleModel::updateBegin, immisciblemodel.hh:278-293):
 * records p_ref = p_w of cell 0 of solution(0). model.update() calls it before every Newton solve
 * (fvbasediscretization.hh:1242); ewg_newton_apply does so itself, and a context that never ran it
 * takes p_ref from solution(0) at its first finite-difference linearization. */
ewg_status ewg_update_begin(ewg_ctx* ctx);
/* The same step with p_ref given by the caller. The reference's updateBegin takes p_w of the first
 * DOF that is local to the process (immisciblemodel.hh:283-291, isLocalDof), so each MPI rank of
 * the reference deflects with its own value. A z-slab of a decomposed grid here passes the whole
 * grid's value instead, p_w of global cell 0, on purpose: its finite-difference deflections, and
 * with them its owned Jacobian rows, then equal the single-domain Jacobian's bit for bit, which a
 * per-slab value would not. p_ref must be positive and finite; it holds until the next
 * ewg_update_begin (ewg_newton_apply runs one). */
ewg_status ewg_set_reference_pressure(ewg_ctx* ctx, double p_ref);

/* linearizeDomain() at the current iterate with time-step size dt: residual r(x) and Jacobian
 * dr/dx into device buffers (fvbaselinearizer.hh:166-197, 401-512). */
ewg_status ewg_linearize(ewg_ctx* ctx, double dt, ewg_lin_report* report);
/* residual() (N x 2, natural order). */
ewg_status ewg_get_residual(ewg_ctx* ctx, double* r);
/* jacobian() as the reference's BCRS: row_ptr[N+1], col_idx[nnzb] (sorted per row), blocks
 * [nnzb][2][2]. Any pointer may be NULL to skip it. */
ewg_status ewg_get_jacobian_bcrs(ewg_ctx* ctx, int32_t* row_ptr, int32_t* col_idx, double* blocks);
/* Intensive quantities of solution(0) per cell, natural order, N x {p_cnw, lambda_w, lambda_n}
 * (ImmiscibleIntensiveQuantities, immiscibleintensivequantities.hh:87-145; lambda = k_r / mu):
 * what VtkMultiPhaseModule writes (io/vtkmultiphasemodule.hh:318-337). */
ewg_status ewg_get_intensive_quantities(ewg_ctx* ctx, double* out);
/* Residual-only evaluation at x (natural order, N x 2) without touching the Jacobian or the
 * stored iterate: max-norm of r(x). Used by the Newton initial-guess fallback. */
ewg_status ewg_residual_norm(ewg_ctx* ctx, const double* x, double dt, double* max_norm);

/* ---- linear solver backend (ParallelBaseBackend::prepare/setResidual/setMatrix/solve) -- */

/* setMatrix(M) from a host BCRS with the structured pattern (same layout as
 * ewg_get_jacobian_bcrs). Overrides the Jacobian of the last linearization. */
ewg_status ewg_set_matrix_bcrs(ewg_ctx* ctx, const int32_t* row_ptr, const int32_t* col_idx,
                               const double* blocks);
/* setResidual(b) (N x 2, natural). Overrides the residual of the last linearization. */
ewg_status ewg_set_residual(ewg_ctx* ctx, const double* b);
/* solve(x): preconditioned BiCGStab on J dx = r, x0 = 0 (parallelbasebackend.hh:301-338,
 * bicgstabsolver.hh:116-326). dx stays on the device; the report carries the outcome.
 * Returns EWG_OK when converged, EWG_ERR_NOT_CONVERGED / EWG_ERR_BREAKDOWN otherwise. */
ewg_status ewg_solve(ewg_ctx* ctx, const ewg_solve_opts* opts, ewg_solve_report* report);
/* The last solution update dx (N x 2, natural). */
ewg_status ewg_get_update(ewg_ctx* ctx, double* dx);
/* Bytes the entry points of this context copied between the caller's host buffers and the device
 * since creation or the last reset (solution, residual, update, matrix and intensive-quantity
 * transfers; the library's own status and norm reads of a few bytes are not counted). reset != 0
 * zeroes the counters after reading. No reference counterpart: it makes the host<->device traffic of
 * a drop-in Newton iteration observable (the reference keeps everything in host memory). */
ewg_status ewg_transfer_counters(ewg_ctx* ctx, int32_t reset, uint64_t* h2d_bytes, uint64_t* d2h_bytes);
/* Apply the preconditioner once, y = M^-1 b (natural order host vectors). For parity tests. */
ewg_status ewg_apply_preconditioner(ewg_ctx* ctx, const ewg_solve_opts* opts, const double* b,
                                    double* y);
/* y = J x with the current Jacobian (natural order host vectors). */
ewg_status ewg_apply_jacobian(ewg_ctx* ctx, const double* x, double* y);

/* ---- device-order vectors (callers that keep their Krylov vectors on the device) --------
 * A device vector is N x 2 doubles in the context's storage order: cell c = i + nx (j + ny k)
 * of colour col = (i + j + k) & 1 sits at entry col * N/2 + c/2, so each z-plane of one colour
 * is a contiguous run of nx*ny/2 entries. Pointers are device memory on the context's device
 * (checked: anything else is EWG_ERR_INVALID), 16-byte aligned; the work is ordered on
 * ewg_get_stream and the calls return without synchronizing. This is the interface of the
 * solve distributed over z-slabs (overlapping Schwarz BiCGStab, parallelbasebackend.hh:301-338
 * with the overlap of overlappingbcrsmatrix.hh). */
typedef enum ewg_buffer {
    EWG_BUFFER_SOLUTION = 0,    /* solution(0), read and written by the caller between calls */
    EWG_BUFFER_RESIDUAL = 1     /* residual of the last linearization */
} ewg_buffer;
/* The device address of one of the context's vectors (valid until ewg_destroy). */
ewg_status ewg_device_buffer(ewg_ctx* ctx, int32_t which, double** out);
/* y = J x with the FP64 Jacobian of the last linearization. */
ewg_status ewg_device_spmv(ewg_ctx* ctx, const double* x, double* y);
/* y = M^-1 b with the preconditioner opts->precond of the last linearization's FP64 Jacobian
 * (factorized at the first call after a linearization). */
ewg_status ewg_device_precondition(ewg_ctx* ctx, const ewg_solve_opts* opts, const double* b,
                                   double* y);
/* Fused kernels of one slab's BiCGStab iteration in a distributed solve (the per-process vector
 * algebra of BiCGStabSolver::apply, bicgstabsolver.hh:207-246, with OverlappingScalarProduct's dot
 * products over the locally owned rows, overlappingscalarproduct.hh:64-80). All vectors are device
 * vectors in this context's storage order (N x 2 doubles); each kernel updates all N rows and
 * reduces over the owned rows only -- rows [own_lo, own_hi) of each of the two colour halves --
 * deterministically into `out`, a device array the caller combines across slabs. The scalars
 * (alpha, omega, beta, the restart flag) are read from `state`, a device BiCGStab state that
 * ewg_device_bicg_state advances from the combined reductions, so no host read is needed between
 * the kernels; once the state has left "running" every kernel returns at once.
 *   bicg_p:         p = r + beta (p - omega v); on a restart r0 = r, v = p = 0 first
 *   bicg_spmv_dot:  y = J x; out[0] = sum_owned w . y          (state may be NULL: no status test)
 *   bicg_hs:        x += alpha y; r -= alpha v; out = {max_owned |r|, max_owned |y|}
 *                   (NaN counts as infinity)
 *   bicg_spmv_dot2: t = J z; out = {t . t, t . s} over owned rows (state may be NULL)
 *   bicg_xr:        x += omega z; out[2..3] = {max |r|, max |z|} with r before its update;
 *                   r -= omega t; out[0..1] = {r0 . r, r . r} over owned rows */
ewg_status ewg_device_bicg_p(ewg_ctx* ctx, double* p, const double* r, double* r0, double* v, const void* state);
ewg_status ewg_device_bicg_spmv_dot(ewg_ctx* ctx, const double* x, double* y, const double* w, int64_t own_lo,
                                    int64_t own_hi, const void* state, double* out);
ewg_status ewg_device_bicg_hs(ewg_ctx* ctx, double* x, const double* y, double* r, const double* v,
                              int64_t own_lo, int64_t own_hi, const void* state, double* out);
ewg_status ewg_device_bicg_spmv_dot2(ewg_ctx* ctx, const double* z, double* t, const double* s, int64_t own_lo,
                                     int64_t own_hi, const void* state, double* out);
ewg_status ewg_device_bicg_xr(ewg_ctx* ctx, double* x, const double* z, double* r, const double* t,
                              const double* r0, int64_t own_lo, int64_t own_hi, const void* state, double* out);
/* The device state of a distributed BiCGStab: ewg_device_bicg_state_size() bytes of device memory
 * the caller owns (one per slab; every slab's copy takes the same steps on the same reductions).
 * ewg_device_bicg_state runs one scalar step on the context's stream, on `red`, the reductions
 * combined over all slabs (device doubles):
 *   stage 0  red = {b.b, max|b|}: CombinedCriterion::setInitial and the top of the first iteration
 *            (tolerances, maximum error and iterations, restart option from opts)
 *   stage 1  red = {r0.v}: alpha = rho_i / r0.v, breakdown tests
 *   stage 2  red = {t.t, t.s, max|s|, max|y|}: the half-step criterion on s (y all zero:
 *            stagnation), omega = t.s / t.t, breakdown tests
 *   stage 3  red = {r0.r, r.r, max|s|, max|z|}: the full-step criterion, the next iteration's top
 *            (restart on breakdown, beta, rho, the iteration limit)
 *   stage 4  red = {r.r, max|r|} of r = b - J x after convergence: resume from x when the true
 *            residual misses the criterion by more than 10x (residual replacement)
 * ewg_device_bicg_state_read copies status (ewg_status-like: 0 running, 1 converged, 2 failed,
 * 3 breakdown, 4 iteration limit), iterations, restarts and the current and initial residual
 * max-norms to the host (one small synchronous read). */
int32_t ewg_device_bicg_state_size(void);
ewg_status ewg_device_bicg_state(ewg_ctx* ctx, int32_t stage, void* state, const double* red,
                                 const ewg_solve_opts* opts);
ewg_status ewg_device_bicg_state_read(ewg_ctx* ctx, const void* state, int32_t* status, int32_t* iterations,
                                      int32_t* restarts, double* residual, double* initial_residual);

/* ---- Newton (NewtonMethod::apply, newtonmethod.hh:308-517) -------------------------- */

/* x(0) -= dx after checking that dx is finite (newtonmethod.hh:743-809). */
ewg_status ewg_newton_update(ewg_ctx* ctx);
/* One full Newton solve of the implicit-Euler step of size dt, starting at solution(0) and with
 * the old storage of solution(1). Mirrors proceed_/preSolve_/update_ exactly; returns EWG_OK if
 * converged. On failure solution(0) holds the last iterate (callers restore it). */
ewg_status ewg_newton_apply(ewg_ctx* ctx, double dt, const ewg_newton_opts* nopts,
                            const ewg_solve_opts* sopts, ewg_newton_report* report);

/* ---- learned Newton initial guess (no reference counterpart; the hook is where the reference
 * copies solution(1) into solution(0), fvbasediscretization.hh:1396-1407 / updateBegin :1311) ---
 *
 * A 4-layer 3x3x3 convolutional network (channels 5 -> 32 -> 32 -> 32 -> 2, ReLU between layers),
 * BF16 weights and activations with FP32 accumulation, trained on the device by its own forward
 * and backward kernels on samples recorded from converged simulator steps. */
typedef struct ewg_net ewg_net;
int64_t ewg_net_num_params(void);
ewg_status ewg_net_create(uint64_t seed, ewg_net** out);
void ewg_net_destroy(ewg_net* net);
const char* ewg_net_last_error(const ewg_net* net);
/* FP32 master parameters: per layer W[27][Cout_pad][Cin_pad] then b[Cout_pad], with Cin_pad
 * 16/32/32/32 and Cout_pad 32/32/32/8 (padded entries are zero). */
ewg_status ewg_net_get_params(ewg_net* net, float* params, int64_t count);
ewg_status ewg_net_set_params(ewg_net* net, const float* params, int64_t count);
/* Input / output normalisation: {p scale, lnK mean, lnK scale, porosity mean, porosity scale,
 * dt scale, dp_w scale, dS_n scale}. */
ewg_status ewg_net_set_scales(ewg_net* net, const double* scales8);
ewg_status ewg_net_get_scales(ewg_net* net, double* scales8);
/* Training loss weights of (dp_w, dS_n) (a saturation weight above 1 also weighs the cells of the
 * plume and its front by that factor), and the guess mode: apply_pressure 0 keeps p_w of the
 * previous solution and applies only the saturation increment, dropping |dS_n| < sn_threshold. */
ewg_status ewg_net_set_options(ewg_net* net, float loss_weight_p, float loss_weight_s, int32_t apply_pressure,
                               double sn_threshold);
/* Forward (and with grads != NULL backward) on host data: features [B][D][H][W][5], targets
 * [..][2] (nullable), outputs [..][2]; loss = mean squared error. For tests and tooling. */
ewg_status ewg_net_eval_host(ewg_net* net, int32_t B, int32_t D, int32_t H, int32_t W, const float* features,
                             const float* targets, float* outputs, float* loss, float* grads);
/* Record the converged step held by ctx (solution(1) -> solution(0), step size dt) as a sample. */
ewg_status ewg_net_record_sample(ewg_net* net, ewg_ctx* ctx, double dt);
int64_t ewg_net_num_samples(const ewg_net* net);
/* Adam steps over the given recorded samples (one sample per step); mean loss out. */
ewg_status ewg_net_train(ewg_net* net, const int64_t* sample_idx, int32_t steps, float lr, float* mean_loss);
ewg_status ewg_net_eval_samples(ewg_net* net, const int64_t* sample_idx, int32_t count, float* mean_loss);
/* Predict solution(0) for the step of size dt from solution(1); keep the prediction only if its
 * residual max-norm does not exceed that of solution(1), else solution(0) = solution(1). */
ewg_status ewg_predict_guess(ewg_ctx* ctx, ewg_net* net, double dt, int32_t* used_guess, double* res_guess,
                             double* res_prev);

/* Forward pass of the guess network that allocates no memory (no reference counterpart). For
 * callers that cannot call cudaMalloc: a host simulator whose own arena owns the device's memory,
 * and step loops that cannot take the device-wide synchronisation of cudaMalloc / cudaFree.
 *   params    device, FP32, the layout of ewg_net_get_params (ewg_net_num_params() floats)
 *   features  device, FP32 [B][D][H][W][5];  outputs  device, FP32 [B][D][H][W][2]
 *   stream    cudaStream_t the work is enqueued on (NULL: the legacy default stream); the call
 *             returns after enqueueing, the outputs are ready once the stream has reached it.
 *   message   optional buffer of message_len bytes for the reason of a failure.
 * The intermediate activations and BF16 weights live in one fixed device array of about 10 MB
 * that every GPU loading this library holds until exit; B*D*H*W above
 * EWG_NET_NOALLOC_MAX_VOXELS is rejected with EWG_ERR_INVALID. The first call on a device looks
 * the array up (cudaGetSymbolAddress) and sets kernel attributes: make that first call before
 * any stream capture. All calls on a device share the array, so calls whose work overlaps on the
 * GPU (different streams, or different host threads) race and corrupt each other's results:
 * order them on one stream. Outputs equal those of ewg_net_eval_host for the same parameters. */
#define EWG_NET_NOALLOC_MAX_VOXELS 65536
ewg_status ewg_net_forward_noalloc(const float* params, int32_t B, int32_t D, int32_t H, int32_t W,
                                   const float* features, float* outputs, void* stream, char* message,
                                   int32_t message_len);

/* One 3x3x3 convolution layer of the guess network on the tensor cores (tcgen05.mma, TMA),
 * synchronous on `stream` (a cudaStream_t; NULL: the default stream). With v a voxel and the
 * taps t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1) over the 27 neighbours (zero outside the volume):
 *   acc[v][o] = sum_t sum_c in[nbr(v, t)][c] w[t][o][c]              (FP32 accumulation)
 *   epilogue 0: out[v][o] = max(acc + bias[o], 0)    epilogue 2: out[v][o] = acc * (mask[v][o] > 0)
 * in: [B][D][H][W][cin] BF16 channels-last, cin 16 or 32; w: [27][32][cin] BF16; bias: 32 FP32
 * (epilogue 0); mask: [B][D][H][W][32] BF16 (epilogue 2); out: [B][D][H][W][32] BF16. Device
 * pointers, 16-byte aligned. EWG_ERR_TIMEOUT: a bounded wait in the kernel gave up. */
ewg_status ewg_net_conv3d(int32_t cin, int32_t epilogue, int32_t B, int32_t D, int32_t H, int32_t W, const void* in,
                          const void* w, const float* bias, const void* mask, void* out, void* stream);

/* ---- batched ensemble (no reference counterpart: the reference runs one lens problem per
 * Simulator; an ensemble of permeability realizations is many such runs of
 * NewtonMethod::apply, newtonmethod.hh:308-517, with FvBaseProblem::timeIntegration's step
 * halving, fvbaseproblem.hh:507-550) ------------------------------------------------------------
 *
 * All members live in one context and share every launch: each kernel covers the tiles of the
 * members in its phase, BiCGStab keeps one state per member and its iterations are replayed from a
 * CUDA graph; each member runs its own Newton iterations and time steps. 3D grids only (even nx),
 * ILU(0) only. */
typedef struct ewg_ensemble ewg_ensemble;

typedef struct ewg_ensemble_opts {
    int32_t precision;       /* EWG_PRECISION_MIXED (default): Jacobian, ILU(0) and BiCGStab of the
                                Newton correction in FP32, residual, update and Newton test in FP64.
                                EWG_PRECISION_FP64: everything in FP64 */
    int32_t use_graph;       /* 1: replay the BiCGStab iterations from a CUDA graph */
    int32_t check_interval;  /* BiCGStab iterations per graph replay / host status read */
    int32_t max_divisions;   /* time-step halvings before a member's step fails (10) */
} ewg_ensemble_opts;

typedef struct ewg_ensemble_report {
    int32_t status;             /* EWG_OK, or the failure of the member's last attempt */
    int32_t newton_iterations;  /* of the accepted attempt */
    int32_t linear_iterations;  /* BiCGStab iterations over all attempts of this step */
    int32_t halvings;           /* step-size halvings before the accepted attempt */
    double dt;                  /* step size of the accepted attempt */
    double error;               /* last Newton error */
} ewg_ensemble_report;

typedef struct ewg_ensemble_stats {
    int32_t rounds;             /* supersteps that linearized at least one member */
    int32_t linear_iterations;  /* BiCGStab iterations summed over members */
    double t_linearize, t_solve, t_update;  /* device seconds per phase */
    double cell_iterations;     /* sum over members of cells x BiCGStab iterations */
    int32_t supersteps;         /* supersteps run (each: linearize, decide, start solves, check_interval
                                   BiCGStab iterations, update) */
} ewg_ensemble_stats;

void ewg_default_ensemble_opts(ewg_ensemble_opts* opts);
/* members problems: grids[m], problems[m] and a natural-order permeability field perms[m]
 * (N_m doubles, borrowed for the call). opts may be NULL (defaults). */
ewg_status ewg_ensemble_create(int32_t members, const ewg_grid* grids, const ewg_problem* problems,
                               const double* const* perms, const ewg_ensemble_opts* opts, ewg_ensemble** out);
void ewg_ensemble_destroy(ewg_ensemble* ens);
const char* ewg_ensemble_last_error(const ewg_ensemble* ens);
const char* ewg_ensemble_create_error(void);
int32_t ewg_ensemble_num_members(const ewg_ensemble* ens);
/* cells of one member; member < 0: all members */
int64_t ewg_ensemble_num_cells(const ewg_ensemble* ens, int32_t member);
void* ewg_ensemble_get_stream(ewg_ensemble* ens);
/* LensProblem::initial into both time levels of every member */
ewg_status ewg_ensemble_apply_initial_solution(ewg_ensemble* ens);
/* solution(time_idx) of one member, natural order N_m x {p_w, S_w} (as ewg_set_solution) */
ewg_status ewg_ensemble_set_solution(ewg_ensemble* ens, int32_t member, int32_t time_idx, const double* x);
ewg_status ewg_ensemble_get_solution(ewg_ensemble* ens, int32_t member, int32_t time_idx, double* x);
/* linearizeDomain() of every member at solution(0) with its own step size dt[m]; the residual
 * max-norm of each member into max_norms[m] (nullable) */
ewg_status ewg_ensemble_linearize(ewg_ensemble* ens, const double* dt, double* max_norms);
/* residual of one member from the last linearization (natural order, N_m x 2) */
ewg_status ewg_ensemble_get_residual(ewg_ensemble* ens, int32_t member, double* r);
/* Launch-shape autotuner: times each kernel class at 1..8 resident blocks per SM (and the
 * assembly's register-budget variants) on the current state with step sizes dt, keeps the fastest.
 * Results do not depend on the choice. */
ewg_status ewg_ensemble_autotune(ewg_ensemble* ens, const double* dt, const ewg_solve_opts* sopts);
/* the chosen blocks per kernel class (count >= 11 entries) and assembly variant */
ewg_status ewg_ensemble_get_launch_shapes(const ewg_ensemble* ens, int32_t* grids, int32_t count,
                                          int32_t* assemble_variant);
/* One implicit-Euler step of every member with its own step size dt[m]: Newton as ewg_newton_apply
 * per member (the same tolerances and iteration rules), a failed attempt restores solution(0) and
 * retries with half the step size, accepted members advance their time level. reports (nullable)
 * receives one entry per member. Returns EWG_OK if every member's step was accepted. */
ewg_status ewg_ensemble_step(ewg_ensemble* ens, const double* dt, const ewg_newton_opts* nopts,
                             const ewg_solve_opts* sopts, ewg_ensemble_report* reports, ewg_ensemble_stats* stats);
/* `steps` implicit steps of every member, each member at its own pace: a member that finishes a
 * Newton iteration or a step goes on at once instead of waiting for the others (the report sums
 * Newton / BiCGStab iterations and halvings over the member's accepted steps). */
ewg_status ewg_ensemble_advance(ewg_ensemble* ens, int32_t steps, const double* dt, const ewg_newton_opts* nopts,
                                const ewg_solve_opts* sopts, ewg_ensemble_report* reports, ewg_ensemble_stats* stats);
/* ewg_ensemble_advance with every Newton, step-size and BiCGStab-stop decision taken on the device:
 * one superstep (linearization, decisions, preconditioner setup, check_interval BiCGStab
 * iterations, Newton update, step acceptance or halving) is the body of a CUDA graph WHILE node,
 * and a launch of that graph runs supersteps until no member is active, reading nothing back to
 * the host; the host reads the scheduler state every 4096 supersteps. Same launches and member
 * sets as ewg_ensemble_advance, so the results are the same bits. stats->t_solve holds the device
 * time of the whole advance (t_linearize and t_update are 0: the phases are not timed apart). */
ewg_status ewg_ensemble_advance_device(ewg_ensemble* ens, int32_t steps, const double* dt,
                                       const ewg_newton_opts* nopts, const ewg_solve_opts* sopts,
                                       ewg_ensemble_report* reports, ewg_ensemble_stats* stats);

/* ---- instrumentation (no reference counterpart; the analogue of the reference's phase timers,
 * newtonmethod.hh:488-500) --------------------------------------------------------------- */

/* The CUDA stream (cudaStream_t) all work of the context is launched on. */
void* ewg_get_stream(ewg_ctx* ctx);
/* Kernel classes: count and names. */
int32_t ewg_profile_num_kernels(void);
const char* ewg_profile_kernel_name(int32_t id);
/* Per-kernel-class device time: with profiling on, launches are bracketed by a CUDA event pair
 * on the context stream: every launch for on == 1, every on-th launch of each class for on > 1
 * (the reported time is then scaled to all launches). Launches are always counted. */
ewg_status ewg_profile_enable(ewg_ctx* ctx, int32_t on);
ewg_status ewg_profile_reset(ewg_ctx* ctx);
ewg_status ewg_profile_get(ewg_ctx* ctx, int32_t id, double* ms_total, int64_t* launches);

/* Default option values of the reference (fvbasediscretization.hh:249-252,
 * parallelbicgstabbackend.hh:48, parallelbasebackend.hh:514, newtonmethod.hh:150-155). */
void ewg_default_solve_opts(ewg_solve_opts* o);
void ewg_default_newton_opts(ewg_newton_opts* o);

/* ---- vertex-centred finite volumes (VcfvDiscretization with UseP1FiniteElementGradients, as
 * tests/lens_immiscible_vcfv_ad.cc selects) ----------------------------------------------------
 *
 * The same model and lens problem with the DOFs at the grid vertices: (nx+1) x (ny+1) [x (nz+1)]
 * vertices, natural order (x fastest), one {p_w, S_w} block per vertex; perm has one value per
 * vertex and the lens region is taken at the vertex positions. Replaces, for the vertex-centred
 * type tag, the Linearizer (fvbaselinearizer.hh:401-512, local residual of
 * discretizations/vcfv/vcfvstencil.hh:866-1016 and p1fegradientcalculator.hh:255-290) and the
 * Newton / BiCGStab path with block ILU(0) or block Jacobi (istlpreconditionerwrappers.hh:145-193).
 * No red-black constraint on nx. */
typedef struct ewg_vcfv ewg_vcfv;

ewg_status ewg_vcfv_create(const ewg_grid* grid, const ewg_problem* problem, const double* perm, ewg_vcfv** out);
void ewg_vcfv_destroy(ewg_vcfv* c);
const char* ewg_vcfv_last_error(const ewg_vcfv* c);
int64_t ewg_vcfv_num_dofs(const ewg_vcfv* c);
/* kernels launched by the context so far */
int64_t ewg_vcfv_launches(const ewg_vcfv* c);
ewg_status ewg_vcfv_set_solution(ewg_vcfv* c, int32_t time_idx, const double* x);
ewg_status ewg_vcfv_get_solution(ewg_vcfv* c, int32_t time_idx, double* x);
/* LensProblem::initial at the vertex positions into solution(0) and solution(1) */
ewg_status ewg_vcfv_apply_initial_solution(ewg_vcfv* c);
ewg_status ewg_vcfv_advance_time_level(ewg_vcfv* c);   /* solution(1) = solution(0) */
ewg_status ewg_vcfv_restore_time_level(ewg_vcfv* c);   /* solution(0) = solution(1) */
/* LocalLinearizerSplice for the vertex-centred stencil: AD (default) or finite differences with
 * NumericDifferenceMethod -1/0/+1 (fvbasefdlocallinearizer.hh; lens_immiscible_vcfv_fd). */
ewg_status ewg_vcfv_set_local_linearizer(ewg_vcfv* c, int32_t kind, int32_t method);
/* ImmiscibleModel::updateBegin: the FD pressure weight's reference pressure (p_w of vertex 0). */
ewg_status ewg_vcfv_update_begin(ewg_vcfv* c);
/* Residual (per unit control volume) and Jacobian of solution(0) against the storage of
 * solution(1); *error = max |r|. */
ewg_status ewg_vcfv_linearize(ewg_vcfv* c, double dt, double* error);
ewg_status ewg_vcfv_get_residual(ewg_vcfv* c, double* r);
/* The Jacobian's 2x2 blocks in the caller's BCRS pattern of the vertex stencil (row v holds the
 * vertices of its adjacent elements, columns ascending). */
ewg_status ewg_vcfv_get_jacobian_bcrs(ewg_vcfv* c, const int32_t* row_ptr, const int32_t* col_idx, int64_t nnzb,
                                      double* blocks);
/* ParallelBaseBackend::solve on the last ewg_vcfv_linearize: BiCGStab for J dx = r with the
 * preconditioner of sopts (as below); dx_out (nullable) receives the update, natural vertex order.
 * EWG_ERR_NOT_CONVERGED when BiCGStab fails, EWG_ERR_BREAKDOWN on breakdown. */
ewg_status ewg_vcfv_solve(ewg_vcfv* c, const ewg_solve_opts* sopts, double* dx_out, int32_t* iterations);
/* NewtonMethod::apply at fixed dt with BiCGStab + block ILU(0) (EWG_PRECOND_ILU0: dune-istl's
 * bilu0 on the matrix ordered by the vertices' parity colour (i&1) + 2 (j&1) + 4 (k&1), then
 * lexicographically) or block Jacobi; FP64 only. */
ewg_status ewg_vcfv_newton_apply(ewg_vcfv* c, double dt, const ewg_newton_opts* nopts, const ewg_solve_opts* sopts,
                                 int32_t* newton_iterations, int32_t* linear_iterations, double* error);

#ifdef __cplusplus
}
#endif

#endif /* EWG_H */
