// TEST PROGRAM: the GPU drop-in headers (GpuEcfvLinearizer, GpuBiCGStabBackend,
// GpuSparseMatrixAdapter) driven by NewtonMethod::apply's exact call sequence
// (nonlinear/newtonmethod.hh:308-517, proceed_ :866-884, preSolve_ :650-685,
// FvBaseNewtonMethod::update_ fvbasenewtonmethod.hh:124-139), compiled against stand-ins of the
// eWoms property system (tests/dropin/ewoms/common/) and of the dune-istl BCRS matrix (below).
//
// Per Newton iteration the caller's side does:
//   linearizer.linearizeDomain(); linearizer.linearizeAuxiliaryEquations();
//   auto& residual = linearizer.residual(); const auto& jacobian = linearizer.jacobian();
//   backend.prepare(jacobian, residual); backend.setResidual(residual); backend.getResidual(residual);
//   error = max |residual|  (preSolve_);  converged -> stop
//   backend.setMatrix(jacobian); update = 0; backend.solve(update);  x = x - update  (update_)
//
// Modes (argv[1]):
//   device  SparseMatrixAdapter = GpuSparseMatrixAdapter: the Jacobian never leaves the device.
//   istl    SparseMatrixAdapter = a host BCRS adapter like IstlSparseMatrixAdapter: the linearizer
//           exports the Jacobian every iteration and the backend uploads it again.
//   host    device mode with a host consumer: after the first linearization the program reads
//           every block through jacobian().block(), scales one diagonal block with setBlock, and
//           solves; the backend uploads the changed matrix. The update is compared with a solve
//           of the same matrix imported through ewg_set_matrix_bcrs on a second context.
// The first two run two implicit steps of a 16 x 12 x 8 lens problem and compare every step
// with ewg_newton_apply on a second context (same Newton iteration counts, same fields bit for
// bit), and print the bytes that crossed between host and device per Newton iteration.
// Output: one "key value" pair per line; the last line is "OK" when every check passed.
#include <ewoms/common/exceptions.hh>
#include <ewoms/common/propertysystem.hh>

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "gpubicgstabbackend.hh"
#include "gpuecfvlinearizer.hh"
#include "gpusparsematrixadapter.hh"

namespace {

int g_failures = 0;
#define CHECK(cond, ...)                                            \
    do {                                                            \
        if (!(cond)) {                                              \
            std::printf("FAIL %s:%d ", __FILE__, __LINE__);         \
            std::printf(__VA_ARGS__);                               \
            std::printf("\n");                                      \
            ++g_failures;                                           \
        }                                                           \
    } while (0)

// ---- stand-ins of Dune::FieldMatrix<double, 2, 2> and Dune::BCRSMatrix (build mode random) ---

struct Block2 {
    using field_type = double;
    double a[2][2];
    Block2() : a{{0, 0}, {0, 0}} {}
    explicit Block2(double v) : a{{v, v}, {v, v}} {}
    double* operator[](int i) { return a[i]; }
    const double* operator[](int i) const { return a[i]; }
    Block2& operator=(double v) { a[0][0] = a[0][1] = a[1][0] = a[1][1] = v; return *this; }
    Block2& operator+=(const Block2& o) {
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) a[i][j] += o.a[i][j];
        return *this;
    }
};

class HostBcrs {
public:
    enum BuildMode { random };

    class Row {
    public:
        class iterator {
        public:
            iterator(HostBcrs* m, size_t q) : m_(m), q_(q) {}
            Block2& operator*() const { return m_->vals_[q_]; }
            Block2* operator->() const { return &m_->vals_[q_]; }
            iterator& operator++() { ++q_; return *this; }
            bool operator!=(const iterator& o) const { return q_ != o.q_; }
            bool operator==(const iterator& o) const { return q_ == o.q_; }
            size_t index() const { return m_->cols_[q_]; }
        private:
            HostBcrs* m_;
            size_t q_;
        };
        Row(HostBcrs* m, size_t r) : m_(m), r_(r) {}
        iterator begin() const { return iterator(m_, m_->rowPtr_[r_]); }
        iterator end() const { return iterator(m_, m_->rowPtr_[r_ + 1]); }
        Block2& operator[](size_t c) const {
            for (size_t q = m_->rowPtr_[r_]; q < m_->rowPtr_[r_ + 1]; ++q)
                if (m_->cols_[q] == c) return m_->vals_[q];
            throw std::out_of_range("HostBcrs: column not in the row's pattern");
        }
    private:
        HostBcrs* m_;
        size_t r_;
    };

    class RowIterator {
    public:
        RowIterator(HostBcrs* m, size_t r) : m_(m), r_(r) {}
        Row* operator->() const { return &m_->rows_[r_]; }
        Row& operator*() const { return m_->rows_[r_]; }
        RowIterator& operator++() { ++r_; return *this; }
        bool operator!=(const RowIterator& o) const { return r_ != o.r_; }
        size_t index() const { return r_; }
    private:
        HostBcrs* m_;
        size_t r_;
    };

    HostBcrs(size_t n, size_t m, BuildMode) : n_(n), m_(m), rowSize_(n, 0) {
        for (size_t r = 0; r < n; ++r) rows_.emplace_back(this, r);
    }
    HostBcrs(const HostBcrs&) = delete;
    void setrowsize(size_t r, size_t s) { rowSize_[r] = s; }
    void endrowsizes() {
        rowPtr_.assign(n_ + 1, 0);
        for (size_t r = 0; r < n_; ++r) rowPtr_[r + 1] = rowPtr_[r] + rowSize_[r];
        cols_.assign(rowPtr_[n_], SIZE_MAX);
        fill_.assign(n_, 0);
        vals_.assign(rowPtr_[n_], Block2(0.0));
    }
    void addindex(size_t r, size_t c) {
        if (c >= m_ || fill_[r] >= rowSize_[r]) throw std::out_of_range("HostBcrs::addindex");
        size_t* row = &cols_[rowPtr_[r]];
        size_t k = fill_[r]++;
        while (k > 0 && row[k - 1] > c) { row[k] = row[k - 1]; --k; }  // keep columns sorted
        row[k] = c;
    }
    void endindices() {}
    HostBcrs& operator=(double v) {
        for (auto& b : vals_) b = v;
        return *this;
    }
    Row& operator[](size_t r) { return rows_[r]; }
    const Row& operator[](size_t r) const { return rows_[r]; }
    RowIterator begin() const { return RowIterator(const_cast<HostBcrs*>(this), 0); }
    RowIterator end() const { return RowIterator(const_cast<HostBcrs*>(this), n_); }
    size_t N() const { return n_; }

private:
    size_t n_, m_;
    std::vector<size_t> rowSize_, rowPtr_, cols_, fill_;
    std::vector<Block2> vals_;
    std::vector<Row> rows_;
};

// a host-memory SparseMatrixAdapter with IstlSparseMatrixAdapter's interface
// (linear/istlsparsematrixadapter.hh:52-165), for the "istl" mode
class HostMatrixAdapter {
public:
    using IstlMatrix = HostBcrs;
    using MatrixBlock = Block2;
    template <class Simulator>
    explicit HostMatrixAdapter(const Simulator& s) : rows_(s.model().numTotalDof()) {}
    template <class Set>
    void reserve(const std::vector<Set>& pattern) {
        m_.reset(new HostBcrs(rows_, rows_, HostBcrs::random));
        for (size_t r = 0; r < rows_; ++r) m_->setrowsize(r, pattern[r].size());
        m_->endrowsizes();
        for (size_t r = 0; r < rows_; ++r)
            for (auto c : pattern[r]) m_->addindex(r, c);
        m_->endindices();
    }
    IstlMatrix& istlMatrix() { return *m_; }
    const IstlMatrix& istlMatrix() const { return *m_; }
    void clear() { (*m_) = 0.0; }
    void addToBlock(size_t r, size_t c, const Block2& b) { (*m_)[r][c] += b; }
    void block(size_t r, size_t c, Block2& b) const { b = (*m_)[r][c]; }

private:
    size_t rows_;
    std::unique_ptr<HostBcrs> m_;
};

// ---- stand-ins of the simulator objects the drop-in headers call ------------------------------

using PrimaryVariables = std::array<double, 2>;
using SolutionVector = std::vector<PrimaryVariables>;

struct Comm {
    int rank() const { return 0; }
    int min(int v) const { return v; }
};
struct StubGridView {
    enum { dimensionworld = 3 };
    const Comm& comm() const { return comm_; }
    Comm comm_;
};
struct StubVanguard {};

// LensProblem's device definition: the 3D lens with a smooth log-normal permeability field
struct StubProblem {
    int nx, ny, nz;
    double lx, ly, lz;
    void gpuProblemDefinition(const StubVanguard&, ewg_problem& p, std::vector<double>& perm) const {
        p = ewg_problem{};
        p.eps = 3e-6; p.porosity = 0.4; p.temperature = 293.15;
        p.rho_w = 1000.0; p.mu_w = 1e-3; p.rho_n = 1460.0; p.mu_n = 5.7e-4;
        p.gravity = 9.81; p.p_ref = 1e5; p.inlet_rate = -0.04;
        const double L[3] = {lx, ly, lz};
        for (int a = 0; a < 3; ++a) { p.lens_lo[a] = 0.3 * L[a]; p.lens_hi[a] = 0.7 * L[a]; }
        p.outer.law = EWG_LAW_VAN_GENUCHTEN; p.outer.swr = 0.05; p.outer.vg_alpha = 3.7e-4; p.outer.vg_n = 4.7;
        p.lens.law = EWG_LAW_VAN_GENUCHTEN; p.lens.swr = 0.18; p.lens.vg_alpha = 4.5e-4; p.lens.vg_n = 7.3;
        p.left_pressure_scale = 1.0;
        p.inlet_x_lo = 2.25 * lx / 6.0; p.inlet_x_hi = 3.75 * lx / 6.0;
        p.inlet_z_lo = 0.3 * lz; p.inlet_z_hi = 0.7 * lz;
        perm.resize((size_t)nx * ny * nz);
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double x = (i + 0.5) * lx / nx, y = (j + 0.5) * ly / ny, z = (k + 0.5) * lz / nz;
                    double lnk = std::log(9.05e-12) + 0.8 * std::sin(1.7 * x + 0.3) * std::cos(2.1 * y) +
                                 0.5 * std::sin(2.9 * z + 1.1 * x);
                    bool lens = x >= p.lens_lo[0] && x <= p.lens_hi[0] && y >= p.lens_lo[1] && y <= p.lens_hi[1] &&
                                z >= p.lens_lo[2] && z <= p.lens_hi[2];
                    if (lens) lnk += std::log(0.1);
                    perm[(size_t)i + (size_t)nx * (j + (size_t)ny * k)] = std::exp(lnk);
                }
    }
};

struct NewtonState {
    unsigned numIt = 0;
    unsigned numIterations() const { return numIt; }
    double tolerance() const { return 1e-8; }
};

template <class TypeTag>
struct StubModel {
    using Linearizer = Ewoms::GpuEcfvLinearizer<TypeTag>;
    SolutionVector sol[2];
    NewtonState newton;
    Linearizer lin;
    size_t n = 0;
    SolutionVector& solution(int t) { return sol[t]; }
    const SolutionVector& solution(int t) const { return sol[t]; }
    NewtonState& newtonMethod() { return newton; }
    const NewtonState& newtonMethod() const { return newton; }
    Linearizer& linearizer() { return lin; }
    const Linearizer& linearizer() const { return lin; }
    size_t numTotalDof() const { return n; }
};

template <class TypeTag>
struct StubSimulator {
    StubModel<TypeTag> model_;
    StubProblem problem_;
    StubVanguard vanguard_;
    StubGridView gridView_;
    double dt = 250.0;
    StubModel<TypeTag>& model() { return model_; }
    const StubModel<TypeTag>& model() const { return model_; }
    const StubProblem& problem() const { return problem_; }
    const StubVanguard& vanguard() const { return vanguard_; }
    const StubGridView& gridView() const { return gridView_; }
    double timeStepSize() const { return dt; }
};

constexpr int NX = 16, NY = 12, NZ = 8;

template <bool DeviceMatrix>
struct TT {
    using Scalar = double;
    using Simulator = StubSimulator<TT>;
    using Model = StubModel<TT>;
    using Problem = StubProblem;
    using SparseMatrixAdapter = typename std::conditional<DeviceMatrix,
        Ewoms::Linear::GpuSparseMatrixAdapter<Block2, HostBcrs>, HostMatrixAdapter>::type;
    using GlobalEqVector = SolutionVector;
    using Constraints = int;
    using GridView = StubGridView;
    struct Params {
        static unsigned CellsX() { return NX; }
        static unsigned CellsY() { return NY; }
        static unsigned CellsZ() { return NZ; }
        static double DomainSizeX() { return 6.0; }
        static double DomainSizeY() { return 4.0; }
        static double DomainSizeZ() { return 3.0; }
        static double LinearSolverTolerance() { return 1e-10; }
        static double LinearSolverAbsTolerance() { return -1.0; }
        static int LinearSolverMaxIterations() { return 1000; }
        static double LinearSolverMaxError() { return 1e7; }
        static double PreconditionerRelaxation() { return 1.0; }
        static std::string GpuPreconditioner() { return "ilu0"; }
        static std::string GpuLinearSolverPrecision() { return "fp64"; }
    };
};

ewg_grid makeGrid() {
    ewg_grid g{};
    g.dim = 3; g.nx = NX; g.ny = NY; g.nz = NZ; g.lx = 6.0; g.ly = 4.0; g.lz = 3.0;
    return g;
}

void pack(const SolutionVector& s, std::vector<double>& out) {
    out.resize(2 * s.size());
    for (size_t i = 0; i < s.size(); ++i) { out[2 * i] = s[i][0]; out[2 * i + 1] = s[i][1]; }
}

struct NewtonResult {
    int iterations = 0;
    bool converged = false;
};

// NewtonMethod::apply's sequence over the drop-in linearizer and backend
template <class Tag>
NewtonResult newtonApply(StubSimulator<Tag>& sim, Ewoms::Linear::GpuBiCGStabBackend<Tag>& backend,
                         unsigned maxIt, std::vector<uint64_t>* h2dPerIt, std::vector<uint64_t>* d2hPerIt) {
    auto& model = sim.model();
    SolutionVector& next = model.solution(0);
    SolutionVector current(next);
    SolutionVector update(next.size());
    auto& lin = model.linearizer();
    const double tol = model.newtonMethod().tolerance();
    double error = 1e100, lastError = 1e100;
    unsigned& numIt = model.newtonMethod().numIt;
    numIt = 0;
    auto proceed = [&]() {
        if (numIt < 1) return true;
        if (error <= tol) return false;
        if (numIt >= maxIt) return error * 4.0 < lastError;
        return true;
    };
    NewtonResult res;
    while (proceed()) {
        current = next;
        lin.linearizeDomain();
        lin.linearizeAuxiliaryEquations();
        auto& residual = lin.residual();
        const auto& jacobian = lin.jacobian();
        backend.prepare(jacobian, residual);
        backend.setResidual(residual);
        backend.getResidual(residual);
        lastError = error;
        error = 0;
        for (const auto& r : residual)
            error = std::max(error, std::max(std::abs(r[0]), std::abs(r[1])));
        if (!proceed()) {
            ++numIt;
            res.converged = error <= tol;
            break;
        }
        backend.setMatrix(jacobian);
        for (auto& u : update) u = {0.0, 0.0};
        if (!backend.solve(update)) return res;
        for (size_t i = 0; i < next.size(); ++i) {
            next[i][0] = current[i][0] - update[i][0];
            next[i][1] = current[i][1] - update[i][1];
        }
        ++numIt;
        if (h2dPerIt) {
            uint64_t h2d = 0, d2h = 0;
            lin.context()->transferCounters(true, &h2d, &d2h);
            h2dPerIt->push_back(h2d);
            d2hPerIt->push_back(d2h);
        }
    }
    res.iterations = (int)numIt;
    return res;
}

template <bool Dev>
void setupSim(StubSimulator<TT<Dev>>& sim, const std::vector<double>& x0) {
    const size_t n = (size_t)NX * NY * NZ;
    sim.problem_ = StubProblem{NX, NY, NZ, 6.0, 4.0, 3.0};
    sim.model_.n = n;
    for (int t = 0; t < 2; ++t) {
        sim.model_.sol[t].resize(n);
        for (size_t i = 0; i < n; ++i) sim.model_.sol[t][i] = {x0[2 * i], x0[2 * i + 1]};
    }
    sim.model_.lin.init(sim);
}

// two implicit steps through the drop-in sequence, each compared with ewg_newton_apply
template <bool Dev>
void runSteps(const char* mode) {
    using Tag = TT<Dev>;
    const size_t n = (size_t)NX * NY * NZ;
    const ewg_grid g = makeGrid();
    StubProblem prob{NX, NY, NZ, 6.0, 4.0, 3.0};
    ewg_problem p;
    std::vector<double> perm;
    prob.gpuProblemDefinition(StubVanguard{}, p, perm);
    ewg::Context ref(g, p, perm);
    ref.applyInitialSolution();
    std::vector<double> x0(2 * n);
    ref.getSolution(0, x0.data());

    StubSimulator<Tag> sim;
    setupSim<Dev>(sim, x0);
    Ewoms::Linear::GpuBiCGStabBackend<Tag> backend(sim);
    ewg_newton_opts no;
    ewg_default_newton_opts(&no);
    ewg_solve_opts so;
    ewg_default_solve_opts(&so);
    so.linear_solver_tolerance = 1e-10;
    so.linear_solver_abs_tolerance = 1e-10;  // NewtonTolerance / 100
    const uint64_t N16 = 16ull * n;
    for (int step = 0; step < 2; ++step) {
        std::vector<uint64_t> h2d, d2h;
        // the counters start with this step: drop what context creation and the last step moved
        if (sim.model_.lin.context()) sim.model_.lin.context()->transferCounters(true, nullptr, nullptr);
        NewtonResult r = newtonApply(sim, backend, no.newton_max_iterations, &h2d, &d2h);
        ewg_newton_report nrep{};
        ewg_status st = ewg_newton_apply(ref.raw(), 250.0, &no, &so, &nrep);
        const int its = nrep.iterations;
        CHECK(st == EWG_OK && r.converged, "step %d: newton failed (%d / %d)", step, (int)st, (int)r.converged);
        CHECK(r.iterations == its, "step %d: drop-in %d Newton iterations, ewg_newton_apply %d", step, r.iterations, its);
        std::vector<double> xd, xr(2 * n);
        pack(sim.model_.sol[0], xd);
        ref.getSolution(0, xr.data());
        double dmax = 0;
        for (size_t i = 0; i < 2 * n; ++i) dmax = std::max(dmax, std::abs(xd[i] - xr[i]));
        CHECK(dmax == 0.0, "step %d: fields differ by %.3e", step, dmax);
        std::printf("%s_step%d_newton_iterations %d\n", mode, step, r.iterations);
        std::printf("%s_step%d_max_field_difference %.3e\n", mode, step, dmax);
        // counters per completed Newton iteration (linearize + solve + update); the first carries
        // the upload of solution(1), and the converging linearization's residual read follows
        for (size_t k = 0; k < h2d.size(); ++k)
            std::printf("%s_step%d_it%zu_h2d_bytes %llu\n%s_step%d_it%zu_d2h_bytes %llu\n", mode, step, k,
                        (unsigned long long)h2d[k], mode, step, k, (unsigned long long)d2h[k]);
        if (Dev) {
            for (size_t k = 0; k < h2d.size(); ++k) {
                const uint64_t expect_h2d = (k == 0 ? 2 : 1) * N16;  // solution(0) (+ solution(1))
                CHECK(h2d[k] == expect_h2d, "step %d it %zu: %llu bytes to the device, expected %llu", step, k,
                      (unsigned long long)h2d[k], (unsigned long long)expect_h2d);
                CHECK(d2h[k] == 2 * N16, "step %d it %zu: %llu bytes to the host, expected %llu (residual + update)",
                      step, k, (unsigned long long)d2h[k], (unsigned long long)(2 * N16));
            }
        }
        // FvBaseDiscretization::advanceTimeLevel: solution(1) = solution(0)
        sim.model_.sol[1] = sim.model_.sol[0];
        ref.advanceTimeLevel();
    }
    if constexpr (Dev) {
        const auto& J = sim.model_.lin.jacobian();
        std::printf("%s_matrix_exports %llu\n%s_matrix_uploads %llu\n", mode, (unsigned long long)J.exports(), mode,
                    (unsigned long long)J.uploads());
        CHECK(J.exports() == 0 && J.uploads() == 0, "device mode moved the matrix");
    }
}

// a host consumer reads and changes blocks of the device-resident Jacobian
void runHostConsumer() {
    using Tag = TT<true>;
    const size_t n = (size_t)NX * NY * NZ;
    const ewg_grid g = makeGrid();
    StubProblem prob{NX, NY, NZ, 6.0, 4.0, 3.0};
    ewg_problem p;
    std::vector<double> perm;
    prob.gpuProblemDefinition(StubVanguard{}, p, perm);
    ewg::Context ref(g, p, perm);
    ref.applyInitialSolution();
    std::vector<double> x0(2 * n);
    ref.getSolution(0, x0.data());
    // a state off the hydrostatic one, so every block is non-trivial
    for (size_t i = 0; i < n; ++i) x0[2 * i + 1] = 1.0 - 0.3 * (double)((i * 2654435761u) % 1000) / 1000.0;

    StubSimulator<Tag> sim;
    setupSim<true>(sim, x0);
    Ewoms::Linear::GpuBiCGStabBackend<Tag> backend(sim);
    auto& lin = sim.model_.lin;
    lin.linearizeDomain();
    auto& J = lin.jacobian();
    CHECK(J.exports() == 0, "linearization exported the matrix");
    // every block through the adapter's host interface equals the C ABI export
    const int64_t nnzb = lin.context()->numBlocks();
    std::vector<int32_t> rp(n + 1), ci(nnzb);
    std::vector<double> blocks(4 * nnzb);
    lin.context()->getJacobianBcrs(rp.data(), ci.data(), blocks.data());
    int mismatches = 0;
    for (size_t r = 0; r < n; ++r)
        for (int32_t q = rp[r]; q < rp[r + 1]; ++q) {
            Block2 b;
            J.block(r, ci[q], b);
            for (int e = 0; e < 2; ++e)
                for (int v = 0; v < 2; ++v) mismatches += b[e][v] != blocks[4 * q + 2 * e + v];
        }
    CHECK(mismatches == 0, "%d host-read entries differ from the export", mismatches);
    CHECK(J.exports() == 1, "host reads exported %llu times (expected once)", (unsigned long long)J.exports());
    // change one diagonal block on the host; setMatrix uploads, solve sees the change
    const size_t row = n / 2;
    Block2 d;
    J.block(row, row, d);
    for (int e = 0; e < 2; ++e)
        for (int v = 0; v < 2; ++v) d[e][v] *= 2.0;
    J.setBlock(row, row, d);
    auto& residual = lin.residual();
    backend.prepare(J, residual);
    backend.setResidual(residual);
    backend.setMatrix(J);
    CHECK(J.uploads() == 1, "setMatrix uploaded %llu times (expected once)", (unsigned long long)J.uploads());
    SolutionVector update(n);
    CHECK(backend.solve(update), "solve of the changed matrix failed");
    // the same matrix and residual imported on a second context through the C ABI
    for (int32_t q = rp[row]; q < rp[row + 1]; ++q)
        if ((size_t)ci[q] == row)
            for (int t = 0; t < 4; ++t) blocks[4 * q + t] *= 2.0;
    std::vector<double> r(2 * n);
    pack(residual, r);
    ewg::Context other(g, p, perm);
    other.setMatrixBcrs(rp.data(), ci.data(), blocks.data());
    other.setResidual(r.data());
    ewg_solve_opts so;
    ewg_default_solve_opts(&so);
    so.linear_solver_tolerance = 1e-10;
    so.linear_solver_abs_tolerance = 1e-10;
    ewg_status st;
    ewg_solve_report rep = other.solve(so, &st);
    CHECK(st == EWG_OK && rep.converged, "reference solve failed");
    std::vector<double> dx(2 * n), du;
    other.getUpdate(dx.data());
    pack(update, du);
    double dmax = 0;
    for (size_t i = 0; i < 2 * n; ++i) dmax = std::max(dmax, std::abs(du[i] - dx[i]));
    CHECK(dmax == 0.0, "updates differ by %.3e", dmax);
    std::printf("host_consumer_max_update_difference %.3e\n", dmax);
    std::printf("host_consumer_matrix_exports %llu\nhost_consumer_matrix_uploads %llu\n",
                (unsigned long long)J.exports(), (unsigned long long)J.uploads());
}

}  // namespace

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "device";
    try {
        if (mode == "device")
            runSteps<true>("device");
        else if (mode == "istl")
            runSteps<false>("istl");
        else if (mode == "host")
            runHostConsumer();
        else {
            std::printf("unknown mode %s\n", mode.c_str());
            return 2;
        }
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        return 1;
    }
    std::printf("cells %d\n", NX * NY * NZ);
    if (g_failures) return 1;
    std::printf("OK\n");
    return 0;
}
