// Ewoms::GpuVcfvLinearizer<TypeTag> and Ewoms::Linear::GpuVcfvBiCGStabBackend<TypeTag>: drop-in
// replacements of FvBaseLinearizer (discretizations/common/fvbaselinearizer.hh) and
// ParallelBiCGStabSolverBackend (linear/parallelbicgstabbackend.hh) for the vertex-centred
// immiscible two-phase model on a structured grid (lens_immiscible_vcfv_ad / _fd), backed by
// libewg.so's ewg_vcfv_* entry points.
//
//   SET_TYPE_PROP(LensProblemVcfvAd, Linearizer, Ewoms::GpuVcfvLinearizer<TypeTag>);
//   SET_TYPE_PROP(LensProblemVcfvAd, LinearSolverBackend, Ewoms::Linear::GpuVcfvBiCGStabBackend<TypeTag>);
//
// The public interfaces are FvBaseLinearizer's and ParallelBaseBackend's, as for the cell-centred
// GpuEcfvLinearizer / GpuBiCGStabBackend. DOFs are the grid vertices in the vertex mapper's
// lexicographic order; the problem provides gpuVertexProblemDefinition(vanguard, ewg_problem&,
// std::vector<double>& permPerVertex). The local linearizer follows LocalLinearizerSplice
// (GpuVcfvUseFiniteDifferences = true selects FiniteDifferenceLocalLinearizer with
// NumericDifferenceMethod). Errors surface as Ewoms::NumericalIssue like fvbaselinearizer.hh:
// 183-196 and bicgstabsolver.hh:196-197. This header compiles inside an eWoms build; it is not
// built in this repository, whose tests drive the same C ABI through ewg.hh and lens_gpu.cc.
#ifndef EWOMS_GPU_VCFV_LINEARIZER_HH
#define EWOMS_GPU_VCFV_LINEARIZER_HH

#include <ewoms/common/exceptions.hh>
#include <ewoms/common/propertysystem.hh>

#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "ewg.hh"

BEGIN_PROPERTIES
NEW_PROP_TAG(GpuVcfvUseFiniteDifferences);
NEW_PROP_TAG(GpuVcfvPreconditioner);
END_PROPERTIES

namespace Ewoms {

template <class TypeTag>
class GpuVcfvLinearizer
{
    using Simulator = GET_PROP_TYPE(TypeTag, Simulator);
    using Scalar = GET_PROP_TYPE(TypeTag, Scalar);
    using SparseMatrixAdapter = GET_PROP_TYPE(TypeTag, SparseMatrixAdapter);
    using GlobalEqVector = GET_PROP_TYPE(TypeTag, GlobalEqVector);
    using Constraints = GET_PROP_TYPE(TypeTag, Constraints);
    using GridView = GET_PROP_TYPE(TypeTag, GridView);
    enum { dimWorld = GridView::dimensionworld };

public:
    GpuVcfvLinearizer() = default;
    GpuVcfvLinearizer(const GpuVcfvLinearizer&) = delete;

    static void registerParameters()
    {
        EWOMS_REGISTER_PARAM(TypeTag, bool, GpuVcfvUseFiniteDifferences,
                             "Linearize with finite differences instead of automatic differentiation");
    }

    void init(Simulator& simulator)
    {
        simulatorPtr_ = &simulator;
        ctx_.reset();
    }

    void eraseMatrix() { jacobianValid_ = false; }

    void linearize()
    {
        linearizeDomain();
        linearizeAuxiliaryEquations();
    }

    // fvbaselinearizer.hh:166-197
    void linearizeDomain()
    {
        int succeeded = 1;
        try {
            if (!ctx_)
                createContext_();
            auto& model = simulatorPtr_->model();
            if (model.newtonMethod().numIterations() == 0) {
                pack_(model.solution(/*timeIdx=*/1), hostX_);
                ctx_->setSolution(1, hostX_.data());
            }
            pack_(model.solution(/*timeIdx=*/0), hostX_);
            ctx_->setSolution(0, hostX_.data());
            ctx_->linearize(simulatorPtr_->timeStepSize());
            ctx_->getResidual(hostR_.data());
            for (size_t i = 0; i < residual_.size(); ++i) {
                residual_[i][0] = hostR_[2 * i];
                residual_[i][1] = hostR_[2 * i + 1];
            }
            jacobianValid_ = false;
        }
        catch (const std::exception& e) {
            std::cout << "rank " << simulatorPtr_->gridView().comm().rank()
                      << " caught an exception while linearizing:" << e.what() << "\n" << std::flush;
            succeeded = 0;
        }
        succeeded = simulatorPtr_->gridView().comm().min(succeeded);
        if (!succeeded)
            throw Ewoms::NumericalIssue("A process did not succeed in linearizing the system");
    }

    void linearizeAuxiliaryEquations() {}
    void finalize() {}

    const SparseMatrixAdapter& jacobian() const { exportJacobian_(); return *jacobian_; }
    SparseMatrixAdapter& jacobian() { exportJacobian_(); return *jacobian_; }
    const GlobalEqVector& residual() const { return residual_; }
    GlobalEqVector& residual() { return residual_; }
    const std::map<unsigned, Constraints>& constraintsMap() const { return constraintsMap_; }

    ewg::VcfvContext* context() const { return ctx_.get(); }

private:
    void createContext_()
    {
        ewg_grid g{};
        g.dim = dimWorld;
        g.nx = EWOMS_GET_PARAM(TypeTag, unsigned, CellsX);
        g.ny = EWOMS_GET_PARAM(TypeTag, unsigned, CellsY);
        g.nz = dimWorld == 3 ? EWOMS_GET_PARAM(TypeTag, unsigned, CellsZ) : 1;
        g.lx = EWOMS_GET_PARAM(TypeTag, Scalar, DomainSizeX);
        g.ly = EWOMS_GET_PARAM(TypeTag, Scalar, DomainSizeY);
        g.lz = dimWorld == 3 ? EWOMS_GET_PARAM(TypeTag, Scalar, DomainSizeZ) : 1.0;
        ewg_problem p{};
        std::vector<double> perm;
        simulatorPtr_->problem().gpuVertexProblemDefinition(simulatorPtr_->vanguard(), p, perm);
        ctx_ = std::make_unique<ewg::VcfvContext>(g, p, perm);
        if (EWOMS_GET_PARAM(TypeTag, bool, GpuVcfvUseFiniteDifferences))
            ctx_->setLocalLinearizer(EWG_LOCAL_LINEARIZER_FD, EWOMS_GET_PARAM(TypeTag, int, NumericDifferenceMethod));
        const size_t n = ctx_->numDofs();
        hostX_.resize(2 * n);
        hostR_.resize(2 * n);
        residual_.resize(n);
        // FvBaseLinearizer::createMatrix_: row v holds the vertices of its adjacent elements
        const int nvx = g.nx + 1, nvy = g.ny + 1, nvz = dimWorld == 3 ? g.nz + 1 : 1;
        rowPtr_.assign(n + 1, 0);
        colIdx_.clear();
        for (int k = 0; k < nvz; ++k)
            for (int j = 0; j < nvy; ++j)
                for (int i = 0; i < nvx; ++i) {
                    for (int dk = (dimWorld == 3 ? -1 : 0); dk <= (dimWorld == 3 ? 1 : 0); ++dk)
                        for (int dj = -1; dj <= 1; ++dj)
                            for (int di = -1; di <= 1; ++di) {
                                const int ii = i + di, jj = j + dj, kk = k + dk;
                                if (ii >= 0 && jj >= 0 && kk >= 0 && ii < nvx && jj < nvy && kk < nvz)
                                    colIdx_.push_back(ii + nvx * (jj + nvy * kk));
                            }
                    rowPtr_[i + nvx * (j + nvy * k) + 1] = (int32_t)colIdx_.size();
                }
    }

    template <class SolutionVector>
    static void pack_(const SolutionVector& sol, std::vector<double>& out)
    {
        for (size_t i = 0; i < sol.size(); ++i) {
            out[2 * i] = sol[i][0];
            out[2 * i + 1] = sol[i][1];
        }
    }

    void exportJacobian_() const
    {
        if (jacobianValid_)
            return;
        const size_t n = rowPtr_.size() - 1;
        std::vector<double> blocks(4 * colIdx_.size());
        ctx_->getJacobianBcrs(rowPtr_.data(), colIdx_.data(), (int64_t)colIdx_.size(), blocks.data());
        if (!jacobian_) {
            std::vector<std::set<unsigned>> pattern(n);
            for (size_t r = 0; r < n; ++r)
                for (int32_t q = rowPtr_[r]; q < rowPtr_[r + 1]; ++q)
                    pattern[r].insert(colIdx_[q]);
            jacobian_.reset(new SparseMatrixAdapter(*simulatorPtr_));
            jacobian_->reserve(pattern);
        }
        jacobian_->clear();
        for (size_t r = 0; r < n; ++r)
            for (int32_t q = rowPtr_[r]; q < rowPtr_[r + 1]; ++q) {
                typename SparseMatrixAdapter::MatrixBlock b;
                b[0][0] = blocks[4 * q]; b[0][1] = blocks[4 * q + 1];
                b[1][0] = blocks[4 * q + 2]; b[1][1] = blocks[4 * q + 3];
                jacobian_->addToBlock(r, colIdx_[q], b);
            }
        jacobianValid_ = true;
    }

    Simulator* simulatorPtr_ = nullptr;
    std::unique_ptr<ewg::VcfvContext> ctx_;
    std::vector<double> hostX_, hostR_;
    std::vector<int32_t> rowPtr_, colIdx_;
    GlobalEqVector residual_;
    mutable std::unique_ptr<SparseMatrixAdapter> jacobian_;
    mutable bool jacobianValid_ = false;
    std::map<unsigned, Constraints> constraintsMap_;
};

namespace Linear {

// ParallelBaseBackend's interface (parallelbasebackend.hh:202-344) on the device system that
// GpuVcfvLinearizer left there; GpuVcfvPreconditioner is ilu0 (default) or jacobi.
template <class TypeTag>
class GpuVcfvBiCGStabBackend
{
    using Simulator = GET_PROP_TYPE(TypeTag, Simulator);
    using Scalar = GET_PROP_TYPE(TypeTag, Scalar);
    using SparseMatrixAdapter = GET_PROP_TYPE(TypeTag, SparseMatrixAdapter);
    using Vector = GET_PROP_TYPE(TypeTag, GlobalEqVector);

public:
    GpuVcfvBiCGStabBackend(const Simulator& simulator) : simulator_(simulator) {}

    static void registerParameters()
    {
        EWOMS_REGISTER_PARAM(TypeTag, std::string, GpuVcfvPreconditioner,
                             "Preconditioner of the device BiCGStab: ilu0 or jacobi");
    }

    void eraseMatrix() {}
    void prepare(const SparseMatrixAdapter&, const Vector&) {}
    void setResidual(const Vector&) {}  // the linearizer wrote it on the device
    void getResidual(Vector&) const {}
    void setMatrix(const SparseMatrixAdapter&) {}

    // ParallelBaseBackend::solve (parallelbasebackend.hh:301-338)
    bool solve(Vector& x)
    {
        ewg_solve_opts o;
        ewg_default_solve_opts(&o);
        o.linear_solver_tolerance = EWOMS_GET_PARAM(TypeTag, Scalar, LinearSolverTolerance);
        o.linear_solver_abs_tolerance = EWOMS_GET_PARAM(TypeTag, Scalar, LinearSolverAbsTolerance);
        if (o.linear_solver_abs_tolerance < 0)
            o.linear_solver_abs_tolerance = simulator_.model().newtonMethod().tolerance() / 100.0;
        o.linear_solver_max_iterations = EWOMS_GET_PARAM(TypeTag, int, LinearSolverMaxIterations);
        o.linear_solver_max_error = EWOMS_GET_PARAM(TypeTag, Scalar, LinearSolverMaxError);
        o.preconditioner_relaxation = EWOMS_GET_PARAM(TypeTag, Scalar, PreconditionerRelaxation);
        o.precond = EWOMS_GET_PARAM(TypeTag, std::string, GpuVcfvPreconditioner) == "jacobi"
            ? EWG_PRECOND_JACOBI : EWG_PRECOND_ILU0;
        host_.resize(2 * x.size());
        int its = 0;
        const ewg_status st = simulator_.model().linearizer().context()->solve(o, host_.data(), &its);
        lastIterations_ = its;
        if (st == EWG_ERR_BREAKDOWN)
            throw Ewoms::NumericalIssue("Breakdown of the BiCGStab solver");
        if (st != EWG_OK)
            return false;
        for (size_t i = 0; i < x.size(); ++i) {
            x[i][0] = host_[2 * i];
            x[i][1] = host_[2 * i + 1];
        }
        return true;
    }

    size_t iterations() const { return lastIterations_; }

private:
    const Simulator& simulator_;
    std::vector<double> host_;
    size_t lastIterations_ = 0;
};

} // namespace Linear
} // namespace Ewoms

#endif
