// C++ host interface over the C ABI of libewg.so (include/ewg.h).
//
// ewg::Context owns one device problem; every failing call throws ewg::Error carrying the
// ewg_status, which eWoms' host code maps to Ewoms::NumericalIssue so FvBaseProblem::
// timeIntegration's time-step halving (fvbaseproblem.hh:507-550) works unchanged.
#ifndef EWG_HOST_EWG_HH
#define EWG_HOST_EWG_HH

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ewg.h"

namespace ewg {

class Error : public std::runtime_error {
public:
    Error(ewg_status st, const std::string& what) : std::runtime_error(what), status_(st) {}
    ewg_status status() const { return status_; }

private:
    ewg_status status_;
};

class Context {
public:
    Context(const ewg_grid& grid, const ewg_problem& problem, const std::vector<double>& perm) {
        ewg_status st = ewg_create(&grid, &problem, perm.data(), &ctx_);
        if (st != EWG_OK) throw Error(st, std::string("ewg_create: ") + ewg_create_error());
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    ~Context() { ewg_destroy(ctx_); }

    ewg_ctx* raw() const { return ctx_; }
    int64_t numCells() const { return ewg_num_cells(ctx_); }
    int64_t numBlocks() const { return ewg_num_blocks(ctx_); }

    void check(ewg_status st, const char* what) const {
        if (st != EWG_OK) throw Error(st, std::string(what) + ": " + ewg_last_error(ctx_));
    }

    void setSolution(int timeIdx, const double* x) { check(ewg_set_solution(ctx_, timeIdx, x), "ewg_set_solution"); }
    void getSolution(int timeIdx, double* x) const { check(ewg_get_solution(ctx_, timeIdx, x), "ewg_get_solution"); }
    void applyInitialSolution() { check(ewg_apply_initial_solution(ctx_), "ewg_apply_initial_solution"); }
    void advanceTimeLevel() { check(ewg_advance_time_level(ctx_), "ewg_advance_time_level"); }
    void restoreTimeLevel() { check(ewg_restore_time_level(ctx_), "ewg_restore_time_level"); }

    void setLocalLinearizer(int kind, int numericDifferenceMethod) {
        check(ewg_set_local_linearizer(ctx_, kind, numericDifferenceMethod), "ewg_set_local_linearizer");
    }
    void updateBegin() { check(ewg_update_begin(ctx_), "ewg_update_begin"); }
    // N x {p_cnw, lambda_w, lambda_n} of solution(0)
    void getIntensiveQuantities(double* out) {
        check(ewg_get_intensive_quantities(ctx_, out), "ewg_get_intensive_quantities");
    }

    ewg_lin_report linearize(double dt) {
        ewg_lin_report rep{};
        check(ewg_linearize(ctx_, dt, &rep), "ewg_linearize");
        return rep;
    }
    void getResidual(double* r) const { check(ewg_get_residual(ctx_, r), "ewg_get_residual"); }
    void getJacobianBcrs(int32_t* rowPtr, int32_t* colIdx, double* blocks) const {
        check(ewg_get_jacobian_bcrs(ctx_, rowPtr, colIdx, blocks), "ewg_get_jacobian_bcrs");
    }
    void setMatrixBcrs(const int32_t* rowPtr, const int32_t* colIdx, const double* blocks) {
        check(ewg_set_matrix_bcrs(ctx_, rowPtr, colIdx, blocks), "ewg_set_matrix_bcrs");
    }
    void setResidual(const double* b) { check(ewg_set_residual(ctx_, b), "ewg_set_residual"); }

    // Returns the report; does not throw on non-convergence (the backend's solve() returns false).
    ewg_solve_report solve(const ewg_solve_opts& o, ewg_status* status) {
        ewg_solve_report rep{};
        *status = ewg_solve(ctx_, &o, &rep);
        if (*status == EWG_ERR_CUDA || *status == EWG_ERR_INVALID || *status == EWG_ERR_TIMEOUT)
            check(*status, "ewg_solve");
        return rep;
    }
    void getUpdate(double* dx) const { check(ewg_get_update(ctx_, dx), "ewg_get_update"); }
    // bytes copied between host buffers and the device by this context's entry points
    void transferCounters(bool reset, uint64_t* h2d, uint64_t* d2h) {
        check(ewg_transfer_counters(ctx_, reset ? 1 : 0, h2d, d2h), "ewg_transfer_counters");
    }
    void newtonUpdate() { check(ewg_newton_update(ctx_), "ewg_newton_update"); }
    double residualNorm(const double* x, double dt) {
        double v = 0;
        check(ewg_residual_norm(ctx_, x, dt, &v), "ewg_residual_norm");
        return v;
    }

private:
    ewg_ctx* ctx_ = nullptr;
};

// The vertex-centred discretization (ewg_vcfv_*): one DOF and one permeability per vertex.
class VcfvContext {
public:
    VcfvContext(const ewg_grid& grid, const ewg_problem& problem, const std::vector<double>& permVertices) {
        ewg_status st = ewg_vcfv_create(&grid, &problem, permVertices.data(), &c_);
        if (st != EWG_OK) throw Error(st, "ewg_vcfv_create failed");
    }
    VcfvContext(const VcfvContext&) = delete;
    VcfvContext& operator=(const VcfvContext&) = delete;
    ~VcfvContext() { ewg_vcfv_destroy(c_); }

    int64_t numDofs() const { return ewg_vcfv_num_dofs(c_); }
    void applyInitialSolution() { check(ewg_vcfv_apply_initial_solution(c_), "ewg_vcfv_apply_initial_solution"); }
    void advanceTimeLevel() { check(ewg_vcfv_advance_time_level(c_), "ewg_vcfv_advance_time_level"); }
    void restoreTimeLevel() { check(ewg_vcfv_restore_time_level(c_), "ewg_vcfv_restore_time_level"); }
    void getSolution(int timeIdx, double* x) { check(ewg_vcfv_get_solution(c_, timeIdx, x), "ewg_vcfv_get_solution"); }
    void setLocalLinearizer(int kind, int method) {
        check(ewg_vcfv_set_local_linearizer(c_, kind, method), "ewg_vcfv_set_local_linearizer");
    }
    void setSolution(int timeIdx, const double* x) { check(ewg_vcfv_set_solution(c_, timeIdx, x), "ewg_vcfv_set_solution"); }
    double linearize(double dt) {
        double err = 0;
        check(ewg_vcfv_linearize(c_, dt, &err), "ewg_vcfv_linearize");
        return err;
    }
    void getResidual(double* r) { check(ewg_vcfv_get_residual(c_, r), "ewg_vcfv_get_residual"); }
    void getJacobianBcrs(const int32_t* rowPtr, const int32_t* colIdx, int64_t nnzb, double* blocks) {
        check(ewg_vcfv_get_jacobian_bcrs(c_, rowPtr, colIdx, nnzb, blocks), "ewg_vcfv_get_jacobian_bcrs");
    }
    // returns the status (EWG_ERR_NOT_CONVERGED / EWG_ERR_BREAKDOWN are the caller's to map)
    ewg_status solve(const ewg_solve_opts& so, double* dx, int* iterations) {
        int32_t it = 0;
        ewg_status st = ewg_vcfv_solve(c_, &so, dx, &it);
        if (iterations) *iterations = it;
        return st;
    }
    // NewtonMethod::apply; returns the status (non-zero: the caller halves the step)
    ewg_status newtonApply(double dt, const ewg_newton_opts& no, const ewg_solve_opts& so, int* its, int* linIts) {
        int32_t a = 0, b = 0;
        double err = 0;
        ewg_status st = ewg_vcfv_newton_apply(c_, dt, &no, &so, &a, &b, &err);
        if (its) *its = a;
        if (linIts) *linIts = b;
        return st;
    }

private:
    void check(ewg_status st, const char* what) {
        if (st != EWG_OK) throw Error(st, std::string(what) + ": " + ewg_vcfv_last_error(c_));
    }
    ewg_vcfv* c_ = nullptr;
};

}  // namespace ewg

#endif
