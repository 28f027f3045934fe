// lens_gpu: the lens_immiscible_ecfv_ad simulation on the B200 path, driven through the C ABI.
//
// Replays the reference's call sequence on top of libewg.so:
//   Ewoms::start / parameter parsing              utils/start.hh:112-199, 273-440
//   Simulator::run time loop                      utils/simulator.hh:660-831
//   FvBaseProblem::timeIntegration (dt halving)   discretizations/common/fvbaseproblem.hh:507-600
//   NewtonMethod::apply / proceed_ / preSolve_    nonlinear/newtonmethod.hh:308-517, 650-685, 866-884
//   NewtonMethod::suggestTimeStepSize             nonlinear/newtonmethod.hh:527-544
// Parameters use the reference's names in kebab case (--end-time=..., --newton-tolerance=...) or a
// --parameter-file=*.ini with Name=value lines; unknown parameters are rejected like the
// reference's parameter system (bin/runtest.sh:262-322).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ewg.hh"
#include "restart.hh"
#include "vtkwriter.hh"

namespace {

struct Params {
    std::map<std::string, std::string> values;
    std::map<std::string, std::string> defaults = {
        {"Preset", "baseline"},        {"GridDim", "2"},
        {"CellsX", "48"},              {"CellsY", "32"},           {"CellsZ", "16"},
        {"DomainSizeX", "6"},          {"DomainSizeY", "4"},        {"DomainSizeZ", "3"},
        {"EndTime", "2500"},           {"InitialTimeStepSize", "250"},
        {"MaxTimeStepSize", "250"},    {"MaxTimeStepDivisions", "10"},
        {"NewtonTolerance", "1e-8"},   {"NewtonMaxIterations", "18"},
        {"NewtonTargetIterations", "10"}, {"NewtonMaxError", "1e100"}, {"NewtonVerbose", "1"},
        {"LinearSolverTolerance", "1e-10"}, {"LinearSolverAbsTolerance", "-1"},
        {"LinearSolverMaxIterations", "1000"}, {"LinearSolverMaxError", "1e7"},
        {"PreconditionerRelaxation", "1"}, {"Preconditioner", "ilu0"},
        {"LinearSolverPrecision", "fp64"}, {"RestartOnBreakdown", "1"},
        {"PermFile", ""},              {"Output", ""},
        {"EnableVtkOutput", "1"},      {"OutputDir", "."},
        {"LocalLinearizer", "ad"},     {"NumericDifferenceMethod", "1"},
        {"Discretization", "ecfv"},
        // Simulator::run restarts from <OutputDir>/<name>_time=<RestartTime>_rank=0.ers when
        // RestartTime > -1e30 (utils/simulator.hh:669-688); a restart file is written after every
        // RestartFileInterval-th time step (FvBaseProblem::shouldWriteRestartFile writes every
        // 10th, fvbaseproblem.hh:611-615; 0: none)
        {"RestartTime", "-1e35"},      {"RestartFileInterval", "10"},
    };
    std::string get(const std::string& k) const {
        auto it = values.find(k);
        return it != values.end() ? it->second : defaults.at(k);
    }
    double d(const std::string& k) const { return std::stod(get(k)); }
    int i(const std::string& k) const { return std::stoi(get(k)); }
};

// --kebab-case-name -> KebabCaseName
std::string camel(const std::string& kebab) {
    std::string out;
    bool up = true;
    for (char c : kebab) {
        if (c == '-') { up = true; continue; }
        out += up ? (char)std::toupper((unsigned char)c) : c;
        up = false;
    }
    return out;
}

void setParam(Params& p, const std::string& name, const std::string& value) {
    if (!p.defaults.count(name)) throw std::runtime_error("unknown parameter '" + name + "'");
    if (p.values.count(name)) throw std::runtime_error("parameter '" + name + "' given twice");
    p.values[name] = value;
}

void parseArgs(int argc, char** argv, Params& p) {
    for (int a = 1; a < argc; ++a) {
        std::string s = argv[a];
        if (s.rfind("--", 0) != 0 || s.find('=') == std::string::npos)
            throw std::runtime_error("malformed argument '" + s + "' (expected --name=value)");
        std::string key = s.substr(2, s.find('=') - 2), val = s.substr(s.find('=') + 1);
        if (key == "parameter-file") {
            std::ifstream f(val);
            if (!f) throw std::runtime_error("parameter file '" + val + "' does not exist");
            std::string line;
            while (std::getline(f, line)) {
                auto hash = line.find('#');
                if (hash != std::string::npos) line = line.substr(0, hash);
                auto eq = line.find('=');
                if (eq == std::string::npos) continue;
                auto trim = [](std::string t) {
                    size_t b = t.find_first_not_of(" \t"), e = t.find_last_not_of(" \t\r");
                    return b == std::string::npos ? std::string() : t.substr(b, e - b + 1);
                };
                setParam(p, trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
            }
            continue;
        }
        setParam(p, camel(key), val);
    }
}

ewg_material vg(double swr, double snr, double alpha, double n) {
    ewg_material m{};
    m.law = EWG_LAW_VAN_GENUCHTEN;
    m.swr = swr; m.snr = snr; m.vg_alpha = alpha; m.vg_n = n;
    return m;
}

// LensProblem::finishInit / boundary constants (lensproblem.hh:248-288, 464-533)
void makeProblem(const Params& p, const ewg_grid& g, ewg_problem& pr, std::vector<double>& perm) {
    pr = ewg_problem{};
    pr.eps = 3e-6;
    pr.porosity = 0.4;
    pr.temperature = 293.15;
    pr.rho_w = 1000.0; pr.mu_w = 1e-3;
    pr.rho_n = 1460.0; pr.mu_n = 5.7e-4;
    pr.gravity = 9.81;
    pr.p_ref = 1e5;
    pr.inlet_rate = -0.04;
    pr.inlet_z_lo = -1e30; pr.inlet_z_hi = 1e30;
    const std::string preset = p.get("Preset");
    double kOuter, kLens;
    if (g.dim == 2) {
        pr.lens_lo[0] = 1.0; pr.lens_lo[1] = 2.0;
        pr.lens_hi[0] = 4.0; pr.lens_hi[1] = 3.0;
    } else {
        for (int a = 0; a < 3; ++a) {
            double L = a == 0 ? g.lx : a == 1 ? g.ly : g.lz;
            pr.lens_lo[a] = 0.3 * L; pr.lens_hi[a] = 0.7 * L;
        }
        pr.inlet_z_lo = 0.3 * g.lz; pr.inlet_z_hi = 0.7 * g.lz;
    }
    if (preset == "reference") {
        pr.outer = vg(0.05, 0.0, 0.0037, 4.7);
        pr.lens = vg(0.18, 0.0, 0.00045, 7.3);
        pr.left_pressure_scale = 1.0 + 1.5 / g.ly;
        pr.inlet_x_lo = 2.0 * g.lx / 6.0; pr.inlet_x_hi = 3.0 * g.lx / 6.0;
        kOuter = 4.6e-10; kLens = 9.05e-12;
    } else if (preset == "baseline") {
        pr.outer = vg(0.05, 0.0, 3.7e-4, 4.7);
        pr.lens = vg(0.18, 0.0, 4.5e-4, 7.3);
        pr.left_pressure_scale = 1.0;
        pr.inlet_x_lo = 2.25 * g.lx / 6.0; pr.inlet_x_hi = 3.75 * g.lx / 6.0;
        kOuter = 9.05e-12; kLens = 9.05e-13;
    } else {
        throw std::runtime_error("unknown preset '" + preset + "' (baseline | reference)");
    }
    const int nz = g.dim == 3 ? g.nz : 1;
    const int64_t N = (int64_t)g.nx * g.ny * nz;
    perm.assign(N, kOuter);
    const std::string permFile = p.get("PermFile");
    if (!permFile.empty()) {
        std::ifstream f(permFile, std::ios::binary);
        if (!f) throw std::runtime_error("cannot open permeability file " + permFile);
        f.read(reinterpret_cast<char*>(perm.data()), sizeof(double) * N);
        if (f.gcount() != (std::streamsize)(sizeof(double) * N))
            throw std::runtime_error("permeability file holds fewer than N doubles");
        return;
    }
    const double h[3] = {g.lx / g.nx, g.ly / g.ny, g.dim == 3 ? g.lz / nz : 1.0};
    for (int64_t c = 0; c < N; ++c) {
        const int64_t idx[3] = {c % g.nx, (c / g.nx) % g.ny, c / ((int64_t)g.nx * g.ny)};
        bool in = true;
        for (int a = 0; a < g.dim; ++a) {
            double x = (idx[a] + 0.5) * h[a];
            if (x < pr.lens_lo[a] - pr.eps || x > pr.lens_hi[a] + pr.eps) in = false;
        }
        if (in) perm[c] = kLens;
    }
}

struct NewtonResult {
    bool converged = false;
    int iterations = 0;
    int linearIterations = 0;
    double tLin = 0, tSolve = 0, tUpdate = 0;
};

// NewtonMethod::apply on top of the low-level C ABI (linearize / solve / update)
NewtonResult newtonApply(ewg::Context& ctx, double dt, const Params& p, const ewg_solve_opts& so) {
    NewtonResult res;
    const double tol = p.d("NewtonTolerance");
    const double maxError = p.d("NewtonMaxError");
    const int maxIt = p.i("NewtonMaxIterations");
    const bool verbose = p.i("NewtonVerbose") != 0;
    int numIterations = 0;
    double error = 1e100, lastError = 1e100;
    auto converged = [&]() { return error <= tol; };
    auto proceed = [&]() {
        if (numIterations < 1) return true;
        if (converged()) return false;
        if (numIterations >= maxIt) return error * 4.0 < lastError;
        return true;
    };
    try {
        while (proceed()) {
            lastError = error;  // beginIteration_
            ewg_lin_report lr = ctx.linearize(dt);
            res.tLin += lr.seconds;
            lastError = error;  // preSolve_
            error = lr.error;
            if (error > maxError) throw ewg::Error(EWG_ERR_MAX_ERROR, "Newton: error above NewtonMaxError");
            if (!proceed()) {
                ++numIterations;
                if (verbose) std::printf("Newton iteration %d error: %g\n", numIterations, error);
                break;
            }
            ewg_status st;
            ewg_solve_report sr = ctx.solve(so, &st);
            res.tSolve += sr.seconds;
            res.linearIterations += sr.iterations;
            if (st != EWG_OK) {
                if (verbose) std::printf("Newton: Linear solver did not converge\n");
                res.iterations = numIterations;
                return res;
            }
            auto t0 = std::chrono::steady_clock::now();
            ctx.newtonUpdate();
            res.tUpdate += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            ++numIterations;
            if (verbose) std::printf("Newton iteration %d error: %g\n", numIterations, error);
        }
    } catch (const ewg::Error& e) {
        if (verbose) std::printf("Newton method caught exception: \"%s\"\n", e.what());
        res.iterations = numIterations;
        return res;
    }
    res.iterations = numIterations;
    res.converged = converged();
    return res;
}

// the fields of VtkMultiPhaseModule for solution(0): pressures, densities, saturations,
// mobilities, relative permeabilities, viscosities, porosity, intrinsic permeability
std::vector<ewg::VtkMultiWriter::Field> vtkFields(ewg::Context& ctx, const ewg_grid& g, const ewg_problem& pr,
                                                  const std::vector<double>& perm) {
    const int64_t N = ctx.numCells();
    std::vector<double> x(2 * N), iq(3 * N);
    ctx.getSolution(0, x.data());
    ctx.getIntensiveQuantities(iq.data());
    using F = ewg::VtkMultiWriter::Field;
    std::vector<F> f = {{"pressure_w", 1, {}}, {"pressure_n", 1, {}}, {"density_w", 1, {}}, {"density_n", 1, {}},
                        {"saturation_w", 1, {}}, {"saturation_n", 1, {}}, {"mobility_w", 1, {}},
                        {"mobility_n", 1, {}}, {"relativePerm_w", 1, {}}, {"relativePerm_n", 1, {}},
                        {"viscosity_w", 1, {}}, {"viscosity_n", 1, {}}, {"porosity", 1, {}},
                        {"intrinsicPerm", g.dim * g.dim, {}}};
    for (auto& fi : f) fi.values.reserve(N * fi.components);
    for (int64_t c = 0; c < N; ++c) {
        const double pw = x[2 * c], sw = x[2 * c + 1], pc = iq[3 * c], lw = iq[3 * c + 1], ln = iq[3 * c + 2];
        const double v[13] = {pw, pw + pc, pr.rho_w, pr.rho_n, sw, 1.0 - sw, lw, ln,
                              lw * pr.mu_w, ln * pr.mu_n, pr.mu_w, pr.mu_n, pr.porosity};
        for (int k = 0; k < 13; ++k) f[k].values.push_back(v[k]);
        for (int r = 0; r < g.dim; ++r)
            for (int q = 0; q < g.dim; ++q) f[13].values.push_back(r == q ? perm[c] : 0.0);
    }
    return f;
}

}  // namespace

// lens_immiscible_vcfv_ad / _fd: the vertex-centred discretization with P1 gradients; BiCGStab
// with block ILU(0) (parity-colour order) or block Jacobi.
// K per vertex from the lens box at the vertex positions (or PermFile with one value per vertex);
// VTK output as point data.
void runVcfv(const Params& p, const ewg_grid& g, const ewg_problem& pr, const std::vector<double>& permCells,
             const ewg_solve_opts& so) {
    (void)permCells;
    const int nz = g.dim == 3 ? g.nz : 1;
    const int nvx = g.nx + 1, nvy = g.ny + 1, nvz = g.dim == 3 ? nz + 1 : 1;
    const int64_t NV = (int64_t)nvx * nvy * nvz;
    const double h[3] = {g.lx / g.nx, g.ly / g.ny, g.dim == 3 ? g.lz / nz : 1.0};
    std::vector<double> perm(NV);
    const std::string permFile = p.get("PermFile");
    if (!permFile.empty()) {
        std::ifstream f(permFile, std::ios::binary);
        if (!f) throw std::runtime_error("cannot open permeability file " + permFile);
        f.read(reinterpret_cast<char*>(perm.data()), sizeof(double) * NV);
        if (f.gcount() != (std::streamsize)(sizeof(double) * NV))
            throw std::runtime_error("permeability file holds fewer values than vertices");
    } else {
        const std::string preset = p.get("Preset");
        const double kOuter = preset == "reference" ? 4.6e-10 : 9.05e-12;
        const double kLens = preset == "reference" ? 9.05e-12 : 9.05e-13;
        for (int64_t v = 0; v < NV; ++v) {
            const int64_t idx[3] = {v % nvx, (v / nvx) % nvy, v / ((int64_t)nvx * nvy)};
            bool in = true;
            for (int a = 0; a < g.dim; ++a) {
                const double x = idx[a] * h[a];
                if (x < pr.lens_lo[a] - pr.eps || x > pr.lens_hi[a] + pr.eps) in = false;
            }
            perm[v] = in ? kLens : kOuter;
        }
    }
    ewg::VcfvContext ctx(g, pr, perm);
    const std::string ll = p.get("LocalLinearizer");
    if (ll != "ad" && ll != "fd") throw std::runtime_error("LocalLinearizer must be 'ad' or 'fd'");
    ctx.setLocalLinearizer(ll == "fd" ? EWG_LOCAL_LINEARIZER_FD : EWG_LOCAL_LINEARIZER_AD, p.i("NumericDifferenceMethod"));
    ctx.applyInitialSolution();
    ewg_newton_opts no;
    ewg_default_newton_opts(&no);
    no.newton_tolerance = p.d("NewtonTolerance");
    no.newton_max_iterations = p.i("NewtonMaxIterations");
    no.newton_max_error = p.d("NewtonMaxError");
    // LensProblem::name(): lens_immiscible_vcfv_ad for AD, lens_immiscible_vcfv for finite differences
    ewg::VtkMultiWriter vtk(p.get("OutputDir"), ll == "ad" ? "lens_immiscible_vcfv_ad" : "lens_immiscible_vcfv");
    const bool vtkOut = p.i("EnableVtkOutput") != 0;
    std::vector<double> x(2 * NV);
    auto fields = [&]() {
        ctx.getSolution(0, x.data());
        std::vector<ewg::VtkMultiWriter::Field> f = {{"pressure_w", 1, {}}, {"saturation_w", 1, {}},
                                                     {"saturation_n", 1, {}}, {"intrinsicPerm", g.dim * g.dim, {}}};
        for (int64_t v = 0; v < NV; ++v) {
            f[0].values.push_back(x[2 * v]);
            f[1].values.push_back(x[2 * v + 1]);
            f[2].values.push_back(1.0 - x[2 * v + 1]);
            for (int r = 0; r < g.dim; ++r)
                for (int c = 0; c < g.dim; ++c) f[3].values.push_back(r == c ? perm[v] : 0.0);
        }
        return f;
    };
    if (vtkOut) vtk.write(0.0, g, fields(), true);
    const double endTime = p.d("EndTime"), maxDt = p.d("MaxTimeStepSize");
    const int maxDivisions = p.i("MaxTimeStepDivisions"), target = p.i("NewtonTargetIterations");
    double t = 0.0, dt = std::min(p.d("InitialTimeStepSize"), maxDt);
    int step = 0;
    auto wall0 = std::chrono::steady_clock::now();
    while (t < endTime * (1 - 1e-12)) {
        dt = std::min(dt, endTime - t);
        int its = 0, lin = 0;
        bool ok = false;
        for (int attempt = 0; attempt < maxDivisions; ++attempt) {
            if (ctx.newtonApply(dt, no, so, &its, &lin) == EWG_OK) { ok = true; break; }
            ctx.restoreTimeLevel();
            std::printf("Newton solver did not converge with dt=%g seconds. Retrying with time step of %g seconds\n",
                        dt, dt / 2.0);
            dt /= 2.0;
        }
        if (!ok) throw std::runtime_error("Newton solver didn't converge after " + std::to_string(maxDivisions) +
                                          " time-step divisions. dt=" + std::to_string(dt));
        ctx.advanceTimeLevel();
        t += dt;
        ++step;
        std::printf("Time step %d done. t=%g s, dt=%g s, Newton iterations %d, linear iterations %d\n", step, t, dt,
                    its, lin);
        if (vtkOut) vtk.write(t, g, fields(), true);
        double next = its > target ? dt / (1.0 + double(its - target) / target)
                                   : dt * (1.0 + double(target - its) / target / 1.2);
        dt = std::min(maxDt, next);
    }
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    std::printf("Simulation of %d time steps took %g seconds\n", step, wall);
    const std::string out = p.get("Output");
    if (!out.empty()) {
        ctx.getSolution(0, x.data());
        std::ofstream f(out, std::ios::binary);
        f.write(reinterpret_cast<const char*>(x.data()), sizeof(double) * x.size());
    }
}

int main(int argc, char** argv) {
    Params p;
    try {
        parseArgs(argc, argv, p);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    try {
        ewg_grid g{};
        g.dim = p.i("GridDim");
        g.nx = p.i("CellsX"); g.ny = p.i("CellsY"); g.nz = g.dim == 3 ? p.i("CellsZ") : 1;
        g.lx = p.d("DomainSizeX"); g.ly = p.d("DomainSizeY"); g.lz = g.dim == 3 ? p.d("DomainSizeZ") : 1.0;
        ewg_problem pr;
        std::vector<double> perm;
        makeProblem(p, g, pr, perm);
        ewg_solve_opts so;
        ewg_default_solve_opts(&so);
        so.linear_solver_tolerance = p.d("LinearSolverTolerance");
        so.linear_solver_abs_tolerance = p.d("LinearSolverAbsTolerance");
        if (so.linear_solver_abs_tolerance < 0) so.linear_solver_abs_tolerance = p.d("NewtonTolerance") / 100.0;
        so.linear_solver_max_iterations = p.i("LinearSolverMaxIterations");
        so.linear_solver_max_error = p.d("LinearSolverMaxError");
        so.preconditioner_relaxation = p.d("PreconditionerRelaxation");
        so.precond = p.get("Preconditioner") == "jacobi" ? EWG_PRECOND_JACOBI : EWG_PRECOND_ILU0;
        so.precision = p.get("LinearSolverPrecision") == "mixed" ? EWG_PRECISION_MIXED : EWG_PRECISION_FP64;
        so.restart_on_breakdown = p.i("RestartOnBreakdown");
        const std::string disc = p.get("Discretization");
        if (disc == "vcfv") {
            runVcfv(p, g, pr, perm, so);
            return 0;
        }
        if (disc != "ecfv") throw std::runtime_error("Discretization must be 'ecfv' or 'vcfv'");
        ewg::Context ctx(g, pr, perm);
        const std::string ll = p.get("LocalLinearizer");
        if (ll != "ad" && ll != "fd") throw std::runtime_error("LocalLinearizer must be 'ad' or 'fd'");
        ctx.setLocalLinearizer(ll == "fd" ? EWG_LOCAL_LINEARIZER_FD : EWG_LOCAL_LINEARIZER_AD,
                               p.i("NumericDifferenceMethod"));
        // LensProblem::name(): lens_<model>_<discretization>[_ad]
        const std::string simName = ll == "ad" ? "lens_immiscible_ecfv_ad" : "lens_immiscible_ecfv";
        ewg::VtkMultiWriter vtk(p.get("OutputDir"), simName);
        const bool vtkOut = p.i("EnableVtkOutput") != 0;
        const int64_t N = ctx.numCells();
        ewg::SimulatorState sim;
        const double restartTime = p.d("RestartTime");
        if (restartTime > -1e30) {
            // Simulator::run: deserialize the simulator, the problem (its VTK writer) and the model
            ewg::Restart res;
            res.deserializeBegin(p.get("OutputDir"), simName, restartTime, g);
            std::printf("Deserialize from file '%s'\n", res.fileNameUsed().c_str());
            res.deserializeSimulator(sim);
            if (vtkOut) {
                int num = 0;
                int64_t pos = 0;
                std::string coll;
                res.deserializeVtkWriter(num, coll, pos);
                vtk.restore(num, coll);
            }
            std::vector<double> x(2 * N);
            res.deserializeCells(x.data(), N);
            res.deserializeEnd();
            ctx.setSolution(0, x.data());
            ctx.setSolution(1, x.data());  // EcfvDiscretization::deserialize: solution(1) = solution(0)
        } else {
            ctx.applyInitialSolution();
            if (vtkOut) vtk.write(0.0, g, vtkFields(ctx, g, pr, perm));
        }
        const double endTime = p.d("EndTime");
        const double maxDt = p.d("MaxTimeStepSize");
        const int maxDivisions = p.i("MaxTimeStepDivisions");
        const int target = p.i("NewtonTargetIterations");
        const int restartInterval = p.i("RestartFileInterval");
        double t = sim.time, dt = std::min(p.d("InitialTimeStepSize"), maxDt);
        int step = sim.timeStepIdx;
        double tLin = 0, tSolve = 0, tUpdate = 0;
        auto wall0 = std::chrono::steady_clock::now();
        while (t < endTime * (1 - 1e-12)) {
            dt = std::min(dt, endTime - t);
            NewtonResult nr;
            bool ok = false;
            for (int attempt = 0; attempt < maxDivisions; ++attempt) {
                ctx.updateBegin();  // model.update() -> updateBegin() before NewtonMethod::apply
                if (so.precision == EWG_PRECISION_MIXED) {
                    // ewg_newton_apply selects the Jacobian precision; the low-level path uses
                    // the FP64 Jacobian, so mixed precision runs through the high-level call
                    ewg_newton_opts no;
                    ewg_default_newton_opts(&no);
                    no.newton_tolerance = p.d("NewtonTolerance");
                    no.newton_max_iterations = p.i("NewtonMaxIterations");
                    ewg_newton_report rep{};
                    ewg_status st = ewg_newton_apply(ctx.raw(), dt, &no, &so, &rep);
                    nr.converged = st == EWG_OK;
                    nr.iterations = rep.iterations;
                    nr.linearIterations = rep.linear_iterations;
                    nr.tLin = rep.t_linearize; nr.tSolve = rep.t_solve; nr.tUpdate = rep.t_update;
                } else {
                    nr = newtonApply(ctx, dt, p, so);
                }
                tLin += nr.tLin; tSolve += nr.tSolve; tUpdate += nr.tUpdate;
                if (nr.converged) { ok = true; break; }
                ctx.restoreTimeLevel();
                std::printf("Newton solver did not converge with dt=%g seconds. Retrying with time step of %g seconds\n",
                            dt, dt / 2.0);
                dt /= 2.0;
            }
            if (!ok) throw std::runtime_error("Newton solver didn't converge after " + std::to_string(maxDivisions) +
                                              " time-step divisions. dt=" + std::to_string(dt));
            ctx.advanceTimeLevel();
            t += dt;
            ++step;
            std::printf("Time step %d done. t=%g s, dt=%g s, Newton iterations %d, linear iterations %d\n",
                        step, t, dt, nr.iterations, nr.linearIterations);
            if (vtkOut) vtk.write(t, g, vtkFields(ctx, g, pr, perm));
            // nextTimeStepSize: min(MaxTimeStepSize, suggestTimeStepSize(dt))
            int n = nr.iterations;
            double next = n > target ? dt / (1.0 + double(n - target) / target)
                                     : dt * (1.0 + double(target - n) / target / 1.2);
            dt = std::min(maxDt, next);
            if (restartInterval > 0 && step > 0 && step % restartInterval == 0) {
                // Simulator::serialize (utils/simulator.hh:923-937)
                sim.time = t;
                sim.timeStepIdx = step;
                ewg::Restart res;
                res.serializeBegin(p.get("OutputDir"), simName, t, g);
                std::printf("Serialize to file '%s', next time step size: %g\n", res.fileNameUsed().c_str(), dt);
                res.serializeSimulator(sim);
                if (vtkOut) res.serializeVtkWriter(vtk.writerNum(), vtk.collection(), vtk.collectionWritePos());
                std::vector<double> x(2 * N);
                ctx.getSolution(0, x.data());
                res.serializeCells(x.data(), N);
                res.serializeEnd();
            }
        }
        double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
        double tot = tLin + tSolve + tUpdate;
        std::printf("Linearization/solve/update time: %g(%g%%)/%g(%g%%)/%g(%g%%)\n", tLin, 100 * tLin / tot, tSolve,
                    100 * tSolve / tot, tUpdate, 100 * tUpdate / tot);
        std::printf("Simulation of %d time steps took %g seconds\n", step, wall);
        const std::string out = p.get("Output");
        if (!out.empty()) {
            std::vector<double> x(2 * ctx.numCells());
            ctx.getSolution(0, x.data());
            std::ofstream f(out, std::ios::binary);
            f.write(reinterpret_cast<const char*>(x.data()), sizeof(double) * x.size());
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
    return 0;
}
