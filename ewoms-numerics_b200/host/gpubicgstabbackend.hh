// Ewoms::Linear::GpuBiCGStabBackend<TypeTag>: drop-in replacement of
// ParallelBiCGStabSolverBackend / ParallelBaseBackend (linear/parallelbicgstabbackend.hh,
// linear/parallelbasebackend.hh) backed by libewg.so.
//
//   SET_TYPE_PROP(LensProblemEcfvAd, LinearSolverBackend, Ewoms::Linear::GpuBiCGStabBackend<TypeTag>);
//
// Interface of ParallelBaseBackend (parallelbasebackend.hh:202-344): ctor(const Simulator&),
// registerParameters, eraseMatrix, prepare, setResidual, getResidual, setMatrix, solve,
// iterations. The runtime parameters keep the reference's names: LinearSolverTolerance,
// LinearSolverAbsTolerance (< 0: NewtonTolerance / 100), LinearSolverMaxIterations,
// LinearSolverMaxError, PreconditionerRelaxation; two are new: GpuPreconditioner (ilu0 | jacobi)
// and GpuLinearSolverPrecision (fp64 | mixed).
//
// The backend solves on the device context of the model's linearizer, which must be
// GpuEcfvLinearizer (it calls linearizer().context()). What setMatrix and setResidual move:
// * setMatrix(M) with the linearizer's GpuSparseMatrixAdapter: nothing, unless a host consumer
//   changed blocks since the linearization, in which case the host copy is uploaded first.
//   Any other SparseMatrixAdapter (IstlSparseMatrixAdapter) is uploaded from M.istlMatrix().
// * setResidual(b) with the linearizer's own residual() object (what NewtonMethod::apply passes,
//   newtonmethod.hh:371-373): nothing, the device residual is the one it was downloaded from.
//   Any other vector is uploaded. getResidual(b) downloads the device residual into any vector
//   but the linearizer's own.
// solve() returns false when BiCGStab does not converge and throws Ewoms::NumericalIssue on
// breakdown, like BiCGStabSolver::apply (bicgstabsolver.hh:196-197, 228-232, 284-288); the update
// is the only vector it downloads. This header compiles inside an eWoms build; the repository
// compiles it against a stand-in of the property system in tests/dropin/.
#ifndef EWOMS_GPU_BICGSTAB_BACKEND_HH
#define EWOMS_GPU_BICGSTAB_BACKEND_HH

#include <ewoms/common/exceptions.hh>
#include <ewoms/common/propertysystem.hh>

#include <string>
#include <vector>

#include "ewg.hh"
#include "gpusparsematrixadapter.hh"

BEGIN_PROPERTIES
NEW_PROP_TAG(GpuPreconditioner);
NEW_PROP_TAG(GpuLinearSolverPrecision);
END_PROPERTIES

namespace Ewoms {
namespace Linear {

template <class TypeTag>
class GpuBiCGStabBackend
{
    using Simulator = GET_PROP_TYPE(TypeTag, Simulator);
    using Scalar = GET_PROP_TYPE(TypeTag, Scalar);
    using SparseMatrixAdapter = GET_PROP_TYPE(TypeTag, SparseMatrixAdapter);
    using Vector = GET_PROP_TYPE(TypeTag, GlobalEqVector);

public:
    GpuBiCGStabBackend(const Simulator& simulator) : simulator_(simulator) {}

    static void registerParameters()
    {
        EWOMS_REGISTER_PARAM(TypeTag, Scalar, LinearSolverTolerance,
                             "The maximum allowed error between of the linear solver");
        EWOMS_REGISTER_PARAM(TypeTag, Scalar, LinearSolverAbsTolerance,
                             "The maximum accepted error of the norm of the residual");
        EWOMS_REGISTER_PARAM(TypeTag, int, LinearSolverMaxIterations,
                             "The maximum number of iterations of the linear solver");
        EWOMS_REGISTER_PARAM(TypeTag, Scalar, LinearSolverMaxError,
                             "The maximum residual error which the linear solver tolerates");
        EWOMS_REGISTER_PARAM(TypeTag, Scalar, PreconditionerRelaxation,
                             "The relaxation factor of the preconditioner");
        EWOMS_REGISTER_PARAM(TypeTag, std::string, GpuPreconditioner,
                             "Preconditioner of the device BiCGStab: ilu0 or jacobi");
        EWOMS_REGISTER_PARAM(TypeTag, std::string, GpuLinearSolverPrecision,
                             "fp64, or mixed: FP32 BiCGStab inside FP64 defect correction");
    }

    void eraseMatrix() {}

    void prepare(const SparseMatrixAdapter&, const Vector&) {}

    void setResidual(const Vector& b)
    {
        if (&b == &simulator_.model().linearizer().residual())
            return;  // downloaded from the device residual by the linearization
        pack_(b, host_);
        ctx_()->setResidual(host_.data());
    }

    void getResidual(Vector& b) const
    {
        if (&b == &simulator_.model().linearizer().residual())
            return;
        host_.resize(2 * b.size());
        ctx_()->getResidual(host_.data());
        for (size_t i = 0; i < b.size(); ++i) {
            b[i][0] = host_[2 * i];
            b[i][1] = host_[2 * i + 1];
        }
    }

    void setMatrix(const SparseMatrixAdapter& M)
    {
        if constexpr (Linear::IsGpuSparseMatrixAdapter<SparseMatrixAdapter>::value) {
            if (M.deviceContext() == ctx_()) {
                // device-resident: upload only what a host consumer changed
                const_cast<SparseMatrixAdapter&>(M).uploadIfHostNewer();
                return;
            }
        }
        const auto& A = M.istlMatrix();
        std::vector<int32_t> rowPtr(A.N() + 1, 0), colIdx;
        std::vector<double> blocks;
        for (auto row = A.begin(); row != A.end(); ++row) {
            for (auto col = row->begin(); col != row->end(); ++col) {
                colIdx.push_back(col.index());
                for (int e = 0; e < 2; ++e)
                    for (int p = 0; p < 2; ++p)
                        blocks.push_back((*col)[e][p]);
            }
            rowPtr[row.index() + 1] = colIdx.size();
        }
        ctx_()->setMatrixBcrs(rowPtr.data(), colIdx.data(), blocks.data());
    }

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
        o.precond = EWOMS_GET_PARAM(TypeTag, std::string, GpuPreconditioner) == "jacobi"
            ? EWG_PRECOND_JACOBI : EWG_PRECOND_ILU0;
        o.precision = EWOMS_GET_PARAM(TypeTag, std::string, GpuLinearSolverPrecision) == "mixed"
            ? EWG_PRECISION_MIXED : EWG_PRECISION_FP64;
        ewg_status st;
        ewg_solve_report rep = ctx_()->solve(o, &st);
        lastIterations_ = rep.iterations;
        if (st == EWG_ERR_BREAKDOWN)
            throw Ewoms::NumericalIssue("Breakdown of the BiCGStab solver");
        if (st != EWG_OK)
            return false;
        host_.resize(2 * x.size());
        ctx_()->getUpdate(host_.data());
        for (size_t i = 0; i < x.size(); ++i) {
            x[i][0] = host_[2 * i];
            x[i][1] = host_[2 * i + 1];
        }
        return true;
    }

    size_t iterations() const { return lastIterations_; }

private:
    ewg::Context* ctx_() const { return simulator_.model().linearizer().context(); }

    static void pack_(const Vector& v, std::vector<double>& out)
    {
        out.resize(2 * v.size());
        for (size_t i = 0; i < v.size(); ++i) {
            out[2 * i] = v[i][0];
            out[2 * i + 1] = v[i][1];
        }
    }

    const Simulator& simulator_;
    mutable std::vector<double> host_;
    size_t lastIterations_ = 0;
};

}} // namespace Linear, Ewoms

#endif
