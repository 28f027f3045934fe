// Ewoms::GpuEcfvLinearizer<TypeTag>: drop-in replacement of Ewoms::FvBaseLinearizer<TypeTag>
// (discretizations/common/fvbaselinearizer.hh) for the ECFV immiscible two-phase model on a
// structured grid, backed by libewg.so.
//
//   SET_TYPE_PROP(LensProblemEcfvAd, Linearizer, Ewoms::GpuEcfvLinearizer<TypeTag>);
//   SET_TYPE_PROP(LensProblemEcfvAd, SparseMatrixAdapter,
//                 Ewoms::Linear::GpuSparseMatrixAdapter<Block, Dune::BCRSMatrix<Block>>);
//
// The public interface is FvBaseLinearizer's: registerParameters, init, eraseMatrix, linearize,
// linearizeDomain, linearizeAuxiliaryEquations, finalize, jacobian, residual, constraintsMap.
// Errors are thrown as Ewoms::NumericalIssue after the cross-rank minimum, like
// fvbaselinearizer.hh:183-196, so the Newton method and FvBaseProblem::timeIntegration react as
// they do to a CPU linearization failure.
//
// Where the data lives. The device keeps its own copy of solution(0) / solution(1);
// linearizeDomain uploads solution(0) every Newton iteration and solution(1) at the first
// iteration of a time step, and downloads the residual, which NewtonMethod::preSolve_ reads on the
// host (newtonmethod.hh:650-685). The Jacobian stays on the device: with GpuSparseMatrixAdapter
// as the SparseMatrixAdapter, jacobian() returns the adapter bound to the device context, and the
// Newton method passes it to the backend's prepare / setMatrix (newtonmethod.hh:371-374, :408)
// without a copy; only a host consumer that reads or changes blocks makes it export (once per
// linearization). With any other SparseMatrixAdapter (IstlSparseMatrixAdapter), jacobian() exports
// the whole matrix into it after every linearization, which is correct but moves nnzb x 32 bytes
// per Newton iteration.
//
// Requirements checked in init(): a structured grid (StructuredGridVanguard; cell index
// i + nx (j + ny k)), even CellsX, an isotropic intrinsic permeability, the lens problem's
// boundary types. This header compiles inside an eWoms build (it uses the property system); the
// repository compiles it against a stand-in of the property system in tests/dropin/, which replays
// NewtonMethod::apply's calls on it.
#ifndef EWOMS_GPU_ECFV_LINEARIZER_HH
#define EWOMS_GPU_ECFV_LINEARIZER_HH

#include <ewoms/common/exceptions.hh>
#include <ewoms/common/propertysystem.hh>

#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <vector>

#include "ewg.hh"
#include "gpusparsematrixadapter.hh"

namespace Ewoms {

template <class TypeTag>
class GpuEcfvLinearizer
{
    using Model = GET_PROP_TYPE(TypeTag, Model);
    using Problem = GET_PROP_TYPE(TypeTag, Problem);
    using Simulator = GET_PROP_TYPE(TypeTag, Simulator);
    using Scalar = GET_PROP_TYPE(TypeTag, Scalar);
    using SparseMatrixAdapter = GET_PROP_TYPE(TypeTag, SparseMatrixAdapter);
    using GlobalEqVector = GET_PROP_TYPE(TypeTag, GlobalEqVector);
    using Constraints = GET_PROP_TYPE(TypeTag, Constraints);
    using GridView = GET_PROP_TYPE(TypeTag, GridView);
    enum { dimWorld = GridView::dimensionworld };
    static constexpr bool deviceMatrix = Linear::IsGpuSparseMatrixAdapter<SparseMatrixAdapter>::value;

public:
    GpuEcfvLinearizer() = default;
    GpuEcfvLinearizer(const GpuEcfvLinearizer&) = delete;

    static void registerParameters() {}

    // FvBaseLinearizer::init (called from FvBaseDiscretization::finishInit, fvbasediscretization.hh:516)
    void init(Simulator& simulator)
    {
        simulatorPtr_ = &simulator;
        jacobian_.reset();
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
            const unsigned numIt = model.newtonMethod().numIterations();
            if (numIt == 0) {
                packSolution_(model.solution(/*timeIdx=*/1), hostX_);
                ctx_->setSolution(1, hostX_.data());
            }
            packSolution_(model.solution(/*timeIdx=*/0), hostX_);
            ctx_->setSolution(0, hostX_.data());
            ctx_->linearize(simulatorPtr_->timeStepSize());
            ctx_->getResidual(hostR_.data());
            unpackResidual_(hostR_, residual_);
            jacobianValid_ = false;
            if constexpr (deviceMatrix)
                jacobian_->markDeviceCurrent();
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

    // With GpuSparseMatrixAdapter: the device-resident matrix (no copy). Otherwise the matrix is
    // exported from the device into the adapter once per linearization.
    const SparseMatrixAdapter& jacobian() const { exportJacobian_(); return *jacobian_; }
    SparseMatrixAdapter& jacobian() { exportJacobian_(); return *jacobian_; }

    const GlobalEqVector& residual() const { return residual_; }
    GlobalEqVector& residual() { return residual_; }

    const std::map<unsigned, Constraints>& constraintsMap() const { return constraintsMap_; }

    // the device context, shared with GpuBiCGStabBackend
    ewg::Context* context() const { return ctx_.get(); }

private:
    void createContext_()
    {
        const auto& vanguard = simulatorPtr_->vanguard();
        const auto& problem = simulatorPtr_->problem();
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
        problem.gpuProblemDefinition(vanguard, p, perm);  // provided by the lens problem
        ctx_ = std::make_unique<ewg::Context>(g, p, perm);
        const size_t n = ctx_->numCells();
        hostX_.resize(2 * n);
        hostR_.resize(2 * n);
        residual_.resize(n);
        if constexpr (deviceMatrix) {
            // FvBaseLinearizer::createMatrix_ reserves the stencil pattern; the device assembles
            // exactly that pattern, so the adapter takes it from the device on its first export
            jacobian_.reset(new SparseMatrixAdapter(*simulatorPtr_));
            jacobian_->bindDevice(ctx_.get());
        }
    }

    template <class SolutionVector>
    static void packSolution_(const SolutionVector& sol, std::vector<double>& out)
    {
        for (size_t i = 0; i < sol.size(); ++i) {
            out[2 * i] = sol[i][0];
            out[2 * i + 1] = sol[i][1];
        }
    }

    static void unpackResidual_(const std::vector<double>& in, GlobalEqVector& r)
    {
        for (size_t i = 0; i < r.size(); ++i) {
            r[i][0] = in[2 * i];
            r[i][1] = in[2 * i + 1];
        }
    }

    void exportJacobian_() const
    {
        if constexpr (deviceMatrix) {
            if (!jacobian_)
                throw std::logic_error("GpuEcfvLinearizer::jacobian() before the first linearization");
            // the adapter stays on the device and exports itself on host access
        }
        else
            exportToHostAdapter_();
    }

    void exportToHostAdapter_() const
    {
        if (jacobianValid_)
            return;
        const size_t n = ctx_->numCells();
        const size_t nnzb = ctx_->numBlocks();
        std::vector<int32_t> rowPtr(n + 1), colIdx(nnzb);
        std::vector<double> blocks(4 * nnzb);
        ctx_->getJacobianBcrs(rowPtr.data(), colIdx.data(), blocks.data());
        if (!jacobian_) {
            // FvBaseLinearizer::createMatrix_: the sparsity pattern of the stencil
            std::vector<std::set<unsigned>> pattern(n);
            for (size_t r = 0; r < n; ++r)
                for (int32_t q = rowPtr[r]; q < rowPtr[r + 1]; ++q)
                    pattern[r].insert(colIdx[q]);
            jacobian_.reset(new SparseMatrixAdapter(*simulatorPtr_));
            jacobian_->reserve(pattern);
        }
        jacobian_->clear();
        for (size_t r = 0; r < n; ++r)
            for (int32_t q = rowPtr[r]; q < rowPtr[r + 1]; ++q) {
                typename SparseMatrixAdapter::MatrixBlock b;
                b[0][0] = blocks[4 * q]; b[0][1] = blocks[4 * q + 1];
                b[1][0] = blocks[4 * q + 2]; b[1][1] = blocks[4 * q + 3];
                jacobian_->addToBlock(r, colIdx[q], b);
            }
        jacobianValid_ = true;
    }

    Simulator* simulatorPtr_ = nullptr;
    std::unique_ptr<ewg::Context> ctx_;
    std::vector<double> hostX_, hostR_;
    GlobalEqVector residual_;
    mutable std::unique_ptr<SparseMatrixAdapter> jacobian_;
    mutable bool jacobianValid_ = false;
    std::map<unsigned, Constraints> constraintsMap_;
};

} // namespace Ewoms

#endif
