/*
 * ewoms_oracle.h -- TEST INFRASTRUCTURE ONLY (the parity checker and the timed CPU baseline).
 *
 * A CPU restatement, in plain C++17, of eWoms' ECFV + forward-mode-AD linearization of the
 * immiscible two-phase model and the BiCGStab / block-ILU0 / block-Jacobi solve it feeds.
 * Nothing in the product links or calls this library; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline arm do.
 *
 * PARITY UNPINNED at the third-party boundary: the reference needs dune-common/geometry/grid/istl,
 * ewoms-common and ewoms-material, none of which exist here, and the reference ships no golden
 * vectors (bin/runtest.sh:144 has the comparison commented out). The material laws
 * (RegularizedVanGenuchten, RegularizedBrooksCorey, EffToAbsLaw), the AD type
 * (DenseAd::Evaluation<double,2>), harmonicMean and dune-istl's block ILU(0) are restated from
 * their published algorithms; everything inside ewoms-numerics is restated from the cited
 * reference lines.
 */
#ifndef EWOMS_ORACLE_H
#define EWOMS_ORACLE_H

#include "../include/ewg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* ordering of the block ILU(0) factorisation */
#define ORC_ORDER_NATURAL 0   /* dune-istl SeqILU on the lexicographic YaspGrid order */
#define ORC_ORDER_REDBLACK 1  /* same factorisation on the red-black permuted matrix */
#define ORC_ORDER_COLOURS 2   /* vertex-centred grids: vertices ordered by the parity colour
                                 (i&1) + 2 (j&1) + 4 (k&1), then lexicographically */
#define ORC_ORDER_BOX8 3      /* 3D cell grids: 2x2x2 boxes in eight colours (bit 1 of i, j, k),
                                 colour-major, boxes (i/4, j/4, k/4) natural, x-fastest inside */

orc_ctx* orc_create(const ewg_grid* grid, const ewg_problem* problem, const double* perm,
                    int nthreads);
void orc_destroy(orc_ctx* c);
const char* orc_last_error(const orc_ctx* c);
int64_t orc_num_cells(const orc_ctx* c);
int64_t orc_num_blocks(const orc_ctx* c);
void orc_set_recycle_first_iteration_storage(orc_ctx* c, int on);

void orc_set_solution(orc_ctx* c, int time_idx, const double* x);
void orc_get_solution(const orc_ctx* c, int time_idx, double* x);
void orc_apply_initial_solution(orc_ctx* c);
void orc_advance_time_level(orc_ctx* c);

/* FvBaseLinearizer::linearizeDomain at solution(0); newton_iteration selects the storage-cache
 * branch (fvbaselocalresidual.hh:538-575). Returns 0 on success. */
int orc_linearize(orc_ctx* c, double dt, int newton_iteration, double* error);
void orc_get_residual(const orc_ctx* c, double* r);
void orc_get_jacobian_bcrs(const orc_ctx* c, int32_t* row_ptr, int32_t* col_idx, double* blocks);
/* Replace the stored Jacobian / residual (to feed a given system to the solver). */
void orc_set_jacobian_blocks(orc_ctx* c, const double* blocks);
void orc_set_residual(orc_ctx* c, const double* r);

/* Forward-difference Jacobian of the oracle residual at solution(0) (the FD local linearizer's
 * idea, fvbasefdlocallinearizer.hh), into BCRS blocks. Used to pin the AD derivatives. */
int orc_fd_jacobian(orc_ctx* c, double dt, double* blocks);

/* Preconditioned BiCGStab (bicgstabsolver.hh:116-326) on the stored system; dx out (natural). */
int orc_solve(orc_ctx* c, const ewg_solve_opts* o, int ordering, double* dx, int* iterations,
              double* final_residual);
int orc_apply_preconditioner(orc_ctx* c, const ewg_solve_opts* o, int ordering, const double* b,
                             double* y);
void orc_apply_jacobian(const orc_ctx* c, const double* x, double* y);

/* NewtonMethod::apply at fixed dt (newtonmethod.hh:308-517). Returns 0 if converged. */
int orc_newton_apply(orc_ctx* c, double dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                     int ordering, int* newton_iterations, int* linear_iterations, double* error);
double orc_residual_norm(orc_ctx* c, const double* x, double dt);

/* Material law of one region at absolute S_w: out = {pcnw, dpcnw/dSw, krw, dkrw/dSw, krn,
 * dkrn/dSw} (EffToAbsLaw over the regularised law, through the AD type). */
void orc_material_eval(const ewg_material* m, double sw, double* out);

/* Sum over cells of the stored storage term phi*S_a*rho_a*V of a time level, per phase. */
void orc_global_storage(const orc_ctx* c, int time_idx, double* out2);
/* Sum of boundary mass rates [kg/s] (positive = out of the domain) at solution(0), per phase. */
void orc_boundary_rates(orc_ctx* c, double* out2);

/* ---- vertex-centred finite volumes (VcfvDiscretization with P1 gradients) ----
 * DOFs at the (nx+1) x (ny+1) [x (nz+1)] vertices, numbered x fastest; perm per vertex. */
typedef struct orc_vcfv orc_vcfv;
orc_vcfv* orc_vcfv_create(const ewg_grid* g, const ewg_problem* p, const double* perm, int nthreads);
void orc_vcfv_destroy(orc_vcfv* c);
const char* orc_vcfv_last_error(const orc_vcfv* c);
int64_t orc_vcfv_num_dofs(const orc_vcfv* c);
int64_t orc_vcfv_num_blocks(const orc_vcfv* c);
void orc_vcfv_set_solution(orc_vcfv* c, int time_idx, const double* x);
void orc_vcfv_get_solution(const orc_vcfv* c, int time_idx, double* x);
void orc_vcfv_apply_initial_solution(orc_vcfv* c);
void orc_vcfv_advance_time_level(orc_vcfv* c);
void orc_vcfv_set_local_linearizer(orc_vcfv* c, int kind, int method);  /* 0 AD, 1 FD */
void orc_vcfv_update_begin(orc_vcfv* c);
void orc_vcfv_total_volumes(const orc_vcfv* c, double* out);
int orc_vcfv_linearize(orc_vcfv* c, double dt, int newton_iteration, double* error);
void orc_vcfv_get_residual(const orc_vcfv* c, double* r);
void orc_vcfv_get_jacobian_bcrs(const orc_vcfv* c, int32_t* row_ptr, int32_t* col_idx, double* blocks);
int orc_vcfv_newton_apply(orc_vcfv* c, double dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                          int ordering, int* newton_iterations, int* linear_iterations, double* error);
void orc_vcfv_global_storage(const orc_vcfv* c, int time_idx, double* out2);
void orc_vcfv_boundary_rates(orc_vcfv* c, double* out2);
void orc_vcfv_geometry(const orc_vcfv* c, int32_t* ij, double* ip, double* nrm, double* area, double* G,
                       double* scv_volume);

#ifdef __cplusplus
}
#endif

#endif
