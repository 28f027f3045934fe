// TEST INFRASTRUCTURE ONLY: parity checker and timed CPU baseline. The product never links this.
//
// CPU restatement of eWoms' ECFV + AD linearization (immiscible two-phase, lens problem) and of
// the BiCGStab / block ILU(0) / block Jacobi solve. The structure follows the reference:
//   element loop, focus = the element's own DOF   fvbaselinearizer.hh:401-512
//   local residual (flux, volume terms, boundary)  fvbaselocalresidual.hh:154-629
//   AD column scatter J[globJ][globI] += dR_j/dx_i fvbaseadlocallinearizer.hh:178-297
//   intensive quantities                           immiscibleintensivequantities.hh:87-145
//   TPFA Darcy flux with gravity and upwinding     darcyfluxmodule.hh:185-527
//   two-point gradients                            fvbasegradientcalculator.hh:194-312
//   free-flow boundary                             immiscibleboundaryratevector.hh:91-153
//   lens problem                                   tests/problems/lensproblem.hh:248-623
//   Newton                                         nonlinear/newtonmethod.hh:308-909
//   BiCGStab + CombinedCriterion                   linear/bicgstabsolver.hh:116-326,
//                                                  linear/combinedcriterion.hh:112-205
// PARITY UNPINNED: the third-party arithmetic (ewoms-material laws, DenseAd, harmonicMean,
// dune-istl ILU) is restated from the published algorithms; no reference binary or golden vector
// exists to pin it.

#include "ewoms_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------------------------
// Forward-mode AD value with two derivatives: restates ewoms-common DenseAd::Evaluation<double,2>
// (value + d/d(p_w), d/d(S_w)); comparisons use the value only.
struct Eval {
    double v = 0.0;
    double d[2] = {0.0, 0.0};
    Eval() = default;
    Eval(double x) : v(x) {}
    static Eval variable(double x, int i) { Eval e(x); e.d[i] = 1.0; return e; }
};
static inline Eval operator+(const Eval& a, const Eval& b) { Eval r; r.v = a.v + b.v; r.d[0] = a.d[0] + b.d[0]; r.d[1] = a.d[1] + b.d[1]; return r; }
static inline Eval operator-(const Eval& a, const Eval& b) { Eval r; r.v = a.v - b.v; r.d[0] = a.d[0] - b.d[0]; r.d[1] = a.d[1] - b.d[1]; return r; }
static inline Eval operator-(const Eval& a) { Eval r; r.v = -a.v; r.d[0] = -a.d[0]; r.d[1] = -a.d[1]; return r; }
static inline Eval operator*(const Eval& a, const Eval& b) {
    Eval r; r.v = a.v * b.v;
    r.d[0] = a.d[0] * b.v + b.d[0] * a.v;
    r.d[1] = a.d[1] * b.v + b.d[1] * a.v;
    return r;
}
static inline Eval operator/(const Eval& a, const Eval& b) {
    // (u/v)' = (v u' - u v') / v^2
    Eval r;
    r.d[0] = (b.v * a.d[0] - a.v * b.d[0]) / (b.v * b.v);
    r.d[1] = (b.v * a.d[1] - a.v * b.d[1]) / (b.v * b.v);
    r.v = a.v / b.v;
    return r;
}
static inline Eval operator+(const Eval& a, double b) { Eval r = a; r.v += b; return r; }
static inline Eval operator+(double a, const Eval& b) { Eval r = b; r.v = a + b.v; return r; }
static inline Eval operator-(const Eval& a, double b) { Eval r = a; r.v -= b; return r; }
static inline Eval operator-(double a, const Eval& b) { Eval r; r.v = a - b.v; r.d[0] = -b.d[0]; r.d[1] = -b.d[1]; return r; }
static inline Eval operator*(const Eval& a, double b) { Eval r; r.v = a.v * b; r.d[0] = a.d[0] * b; r.d[1] = a.d[1] * b; return r; }
static inline Eval operator*(double a, const Eval& b) { Eval r; r.v = a * b.v; r.d[0] = a * b.d[0]; r.d[1] = a * b.d[1]; return r; }
static inline Eval operator/(const Eval& a, double b) { Eval r; r.v = a.v / b; r.d[0] = a.d[0] / b; r.d[1] = a.d[1] / b; return r; }
static inline Eval operator/(double a, const Eval& b) {
    Eval r; r.v = a / b.v;
    r.d[0] = -a * b.d[0] / (b.v * b.v);
    r.d[1] = -a * b.d[1] / (b.v * b.v);
    return r;
}
static inline Eval& operator+=(Eval& a, const Eval& b) { a = a + b; return a; }
static inline Eval& operator-=(Eval& a, const Eval& b) { a = a - b; return a; }
static inline Eval& operator*=(Eval& a, const Eval& b) { a = a * b; return a; }
static inline Eval& operator/=(Eval& a, double b) { a = a / b; return a; }
static inline Eval pow(const Eval& x, double e) {
    Eval r;
    double px = std::pow(x.v, e);
    if (x.v == 0.0) return Eval(0.0);  // DenseAd special-cases base 0
    double df = px / x.v * e;
    r.v = px; r.d[0] = df * x.d[0]; r.d[1] = df * x.d[1];
    return r;
}
static inline Eval sqrt(const Eval& x) {
    Eval r; double s = std::sqrt(x.v); double df = 0.5 / s;
    r.v = s; r.d[0] = df * x.d[0]; r.d[1] = df * x.d[1];
    return r;
}
static inline double val(const Eval& e) { return e.v; }
static inline double val(double e) { return e; }
static inline double pow(double x, double e) { return std::pow(x, e); }
static inline double sqrt(double x) { return std::sqrt(x); }

// ewoms-common harmonicMean: 0 if x*y <= 0, else 2xy/(y+x)
static inline double harmonicMean(double x, double y) {
    if (x * y <= 0) return 0.0;
    return (2 * x * y) / (y + x);
}

// ---------------------------------------------------------------------------------------------
// Material laws (ewoms-material, restated). One region's parameters, finalized like
// RegularizedVanGenuchtenParams::finalize / RegularizedBrooksCoreyParams.
struct Law {
    int kind = EWG_LAW_VAN_GENUCHTEN;
    double swr = 0, snr = 0;
    // van Genuchten
    double alpha = 0, n = 0, m = 0;
    double pcLowSw = 0.01, pcHighSw = 0.99;
    double pcLow = 0, pcSlopeLow = 0, pcHigh = 0, pcSlopeHigh = 0;
    double spX0 = 0, spX1 = 1, spY0 = 0, spY1 = 0, spM0 = 0, spM1 = 0;
    // Brooks-Corey
    double pe = 0, lambda = 0;
};

template <class E> static E vgPcnw(const Law& p, const E& Sw) {
    return pow(pow(Sw, -1.0 / p.m) - 1.0, 1.0 / p.n) / p.alpha;
}
template <class E> static E vgKrw(const Law& p, const E& Sw) {
    E r = 1.0 - pow(1.0 - pow(Sw, 1.0 / p.m), p.m);
    return sqrt(Sw) * r * r;
}
template <class E> static E vgKrn(const Law& p, const E& Sw) {
    return pow(1.0 - Sw, 1.0 / 3) * pow(1.0 - pow(Sw, 1.0 / p.m), 2 * p.m);
}
// cubic Hermite segment through (x0,y0,m0), (x1,y1,m1): a two-point spline with given slopes
template <class E> static E hermite(const Law& p, const E& x) {
    double h = p.spX1 - p.spX0;
    E t = (x - p.spX0) / h;
    E t2 = t * t;
    E t3 = t2 * t;
    E h00 = 2.0 * t3 - 3.0 * t2 + 1.0;
    E h10 = t3 - 2.0 * t2 + t;
    E h01 = -2.0 * t3 + 3.0 * t2;
    E h11 = t3 - t2;
    return h00 * p.spY0 + h10 * (h * p.spM0) + h01 * p.spY1 + h11 * (h * p.spM1);
}
template <class E> static E regVgPcnw(const Law& p, const E& Sw) {
    if (val(Sw) < p.pcLowSw) return p.pcLow + p.pcSlopeLow * (Sw - p.pcLowSw);
    if (val(Sw) > p.pcHighSw) {
        double yTh = p.pcHigh;
        double m1 = (0.0 - yTh) / (1.0 - p.pcHighSw) * 2;
        if (val(Sw) < 1.0) return hermite(p, Sw);
        return m1 * (Sw - 1.0) + 0.0;
    }
    return vgPcnw(p, Sw);
}
template <class E> static E regVgKrw(const Law& p, const E& Sw) {
    if (val(Sw) <= 0) return E(0.0);
    if (val(Sw) >= 1) return E(1.0);
    return vgKrw(p, Sw);
}
template <class E> static E regVgKrn(const Law& p, const E& Sw) {
    if (val(Sw) <= 0) return E(1.0);
    if (val(Sw) >= 1) return E(0.0);
    return vgKrn(p, Sw);
}
static double bcDPc(const Law& p, double Sw) { return -p.pe / p.lambda * std::pow(Sw, -1.0 / p.lambda - 1.0); }
template <class E> static E regBcPcnw(const Law& p, const E& Sw) {
    const double th = p.pcLowSw;
    if (val(Sw) <= th) {
        double m = bcDPc(p, th);
        double pcTh = p.pe * std::pow(th, -1.0 / p.lambda);
        return pcTh + m * (Sw - th);
    }
    if (val(Sw) >= 1.0) {
        double m = bcDPc(p, 1.0);
        return p.pe + m * (Sw - 1.0);
    }
    return p.pe * pow(Sw, -1.0 / p.lambda);
}
template <class E> static E regBcKrw(const Law& p, const E& Sw) {
    if (val(Sw) <= 0) return E(0.0);
    if (val(Sw) >= 1) return E(1.0);
    return pow(Sw, 2.0 / p.lambda + 3);
}
template <class E> static E regBcKrn(const Law& p, const E& Sw) {
    if (val(Sw) >= 1) return E(0.0);
    if (val(Sw) <= 0) return E(1.0);
    return pow(1.0 - Sw, 2) * (1.0 - pow(Sw, 2.0 / p.lambda + 1));
}
// RegularizedVanGenuchtenParams::dPcnw_dSw_: central finite difference, eps 1e-7
static double vgDPcFd(const Law& p, double Sw) {
    const double eps = 1e-7;
    double delta = 0.0, pc1, pc2;
    if (Sw + eps < 1.0) { pc2 = vgPcnw(p, Sw + eps); delta += eps; } else pc2 = vgPcnw(p, Sw);
    if (Sw - eps > 0.0) { pc1 = vgPcnw(p, Sw - eps); delta += eps; } else pc1 = vgPcnw(p, Sw);
    return (pc2 - pc1) / delta;
}
static Law makeLaw(const ewg_material& m) {
    Law p;
    p.kind = m.law;
    p.swr = m.swr; p.snr = m.snr;
    if (m.law == EWG_LAW_VAN_GENUCHTEN) {
        p.alpha = m.vg_alpha; p.n = m.vg_n; p.m = 1.0 - 1.0 / m.vg_n;
        p.pcLowSw = 0.01; p.pcHighSw = 0.99;
        p.pcLow = vgPcnw(p, p.pcLowSw);
        p.pcSlopeLow = vgDPcFd(p, p.pcLowSw);
        p.pcHigh = vgPcnw(p, p.pcHighSw);
        p.pcSlopeHigh = 2 * (0.0 - p.pcHigh) / (1.0 - p.pcHighSw);
        double mTh = vgDPcFd(p, p.pcHighSw);
        p.spX0 = p.pcHighSw; p.spX1 = 1.0; p.spY0 = p.pcHigh; p.spY1 = 0.0;
        p.spM0 = mTh; p.spM1 = p.pcSlopeHigh;
    } else {
        p.pe = m.bc_entry_pressure; p.lambda = m.bc_lambda; p.pcLowSw = 0.01;
    }
    return p;
}
// EffToAbsLaw: effective saturation (S - Sr)/(1 - sum Sr); krn reads 1 - S_n,eff
template <class E> static void capillaryPressures(E pc[2], const Law& p, const E& Sw) {
    E Se = (Sw - p.swr) / (1.0 - (p.swr + p.snr));
    pc[0] = E(0.0);
    pc[1] = (p.kind == EWG_LAW_VAN_GENUCHTEN) ? regVgPcnw(p, Se) : regBcPcnw(p, Se);
}
template <class E> static void relativePermeabilities(E kr[2], const Law& p, const E& Sw) {
    E Sn = 1.0 - Sw;
    E Sew = (Sw - p.swr) / (1.0 - (p.swr + p.snr));
    E Sen = (Sn - p.snr) / (1.0 - (p.swr + p.snr));
    E Swn = 1.0 - Sen;
    if (p.kind == EWG_LAW_VAN_GENUCHTEN) { kr[0] = regVgKrw(p, Sew); kr[1] = regVgKrn(p, Swn); }
    else { kr[0] = regBcKrw(p, Sew); kr[1] = regBcKrn(p, Swn); }
}

// ---------------------------------------------------------------------------------------------
struct IQ {  // ImmiscibleIntensiveQuantities
    Eval p[2], S[2], rho[2], mu[2], kr[2], mob[2];
    double porosity = 0, K = 0;
};

struct Face {            // one intersection of a cell (YaspGrid order: -x,+x,-y,+y,-z,+z)
    int axis, side;      // side 0: lower face (normal -e_axis), 1: upper face
    int64_t nbr;         // neighbour cell or -1 on the boundary
};

struct Ctx {
    int dim = 2, n[3] = {1, 1, 1};
    double L[3] = {1, 1, 1}, h[3] = {1, 1, 1};
    int64_t N = 0;
    ewg_problem prob{};
    Law law[2];                      // 0 outer, 1 lens
    std::vector<double> perm;
    std::vector<unsigned char> inLens;
    std::vector<double> sol[2];      // solution(timeIdx), N x 2
    std::vector<double> storageOld;  // cached storage of timeIdx 1 (per unit volume), N x 2
    std::vector<double> resid;       // N x 2
    std::vector<int32_t> rowPtr, colIdx;
    std::vector<double> blocks;      // nnzb x 4
    std::vector<IQ> iqCache;
    bool recycleStorage = true;
    // LocalLinearizerSplice: false = AutoDiffLocalLinearizer, true = FiniteDifferenceLocalLinearizer
    // with NumericDifferenceMethod fdMethod (-1 backward, 0 central, +1 forward) and the reference
    // pressure of ImmiscibleModel::updateBegin for the pressure weight (immisciblemodel.hh:278-310)
    bool fd = false;
    int fdMethod = 1;
    double refPressure = -1.0;  // unset until updateBegin
    int nthreads = 1;
    std::string err;

    double vol() const { return dim == 2 ? h[0] * h[1] : h[0] * h[1] * h[2]; }
    double area(int axis) const {
        if (dim == 2) return axis == 0 ? h[1] : h[0];
        return axis == 0 ? h[1] * h[2] : (axis == 1 ? h[0] * h[2] : h[0] * h[1]);
    }
    void ijk(int64_t c, int64_t& i, int64_t& j, int64_t& k) const {
        i = c % n[0]; j = (c / n[0]) % n[1]; k = c / ((int64_t)n[0] * n[1]);
    }
    // global plane index of plane 0: a z-slab of a decomposed grid keeps the global coordinates
    int64_t kOrigin = 0;
    void center(int64_t c, double x[3]) const {
        int64_t id[3]; ijk(c, id[0], id[1], id[2]);
        id[2] += kOrigin;
        for (int a = 0; a < 3; ++a) x[a] = (a < dim) ? (id[a] + 0.5) * h[a] : 0.0;
    }
    void faceCenter(int64_t c, int axis, int side, double x[3]) const {
        int64_t id[3]; ijk(c, id[0], id[1], id[2]);
        id[2] += kOrigin;
        center(c, x);
        x[axis] = (id[axis] + side) * h[axis];
    }
    int numFaces() const { return 2 * dim; }
    void faces(int64_t c, Face f[6]) const {
        int64_t id[3]; ijk(c, id[0], id[1], id[2]);
        int64_t stride[3] = {1, n[0], (int64_t)n[0] * n[1]};
        for (int a = 0; a < dim; ++a)
            for (int s = 0; s < 2; ++s) {
                Face& F = f[2 * a + s];
                F.axis = a; F.side = s;
                bool has = s == 0 ? id[a] > 0 : id[a] < n[a] - 1;
                F.nbr = has ? c + (s == 0 ? -stride[a] : stride[a]) : -1;
            }
    }
    bool isInLens(const double x[3]) const {
        for (int a = 0; a < dim; ++a)
            if (x[a] < prob.lens_lo[a] - prob.eps || x[a] > prob.lens_hi[a] + prob.eps) return false;
        return true;
    }
    double gravity(int a) const { return a == 1 ? -prob.gravity : 0.0; }
};

static IQ computeIQAt(const Ctx& C, int64_t c, double pw, double sw, bool variable) {
    IQ q;
    const Law& L = C.law[C.inLens[c]];
    Eval Sw = variable ? Eval::variable(sw, 1) : Eval(sw);
    q.S[0] = Sw;
    q.S[1] = 1.0 - (Eval(0.0) + Sw);
    Eval pC[2];
    capillaryPressures(pC, L, q.S[0]);
    relativePermeabilities(q.kr, L, q.S[0]);
    Eval p0 = variable ? Eval::variable(pw, 0) : Eval(pw);
    for (int a = 0; a < 2; ++a) q.p[a] = p0 + (pC[a] - pC[0]);
    q.mu[0] = Eval(C.prob.mu_w); q.mu[1] = Eval(C.prob.mu_n);
    q.rho[0] = Eval(C.prob.rho_w); q.rho[1] = Eval(C.prob.rho_n);
    for (int a = 0; a < 2; ++a) q.mob[a] = q.kr[a] / q.mu[a];
    q.porosity = C.prob.porosity;
    q.K = C.perm[c];
    return q;
}
static IQ computeIQ(const Ctx& C, int64_t c, const double* x, bool variable) {
    return computeIQAt(C, c, x[2 * c + 0], x[2 * c + 1], variable);
}

// ImmiscibleLocalResidual::computeStorage: phi * S_a * rho_a
template <class E> static void storageOf(const IQ& q, E out[2]);
template <> void storageOf<Eval>(const IQ& q, Eval out[2]) {
    for (int a = 0; a < 2; ++a) out[a] = Eval(q.porosity) * q.S[a] * q.rho[a];
}
template <> void storageOf<double>(const IQ& q, double out[2]) {
    for (int a = 0; a < 2; ++a) out[a] = q.porosity * q.S[a].v * q.rho[a].v;
}

// Interior-face flux (mass per area) seen from the focus cell i = interior DOF (ECFV: focus is
// always the element's own DOF): darcyfluxmodule.hh:185-324, 461-527, immisciblelocalresidual.hh:123-149.
static void interiorFlux(const Ctx& C, int64_t ci, int64_t cj, const Face& f, const IQ& qi,
                         const IQ& qj, Eval flux[2]) {
    double xi[3], xj[3], xf[3];
    C.center(ci, xi); C.center(cj, xj); C.faceCenter(ci, f.axis, f.side, xf);
    double nrm[3] = {0, 0, 0};
    nrm[f.axis] = f.side == 0 ? -1.0 : 1.0;
    const int dim = C.dim;
    double distSq = 0.0;
    for (int d = 0; d < dim; ++d) { double t = xj[d] - xi[d]; distSq += t * t; }
    Eval grad[2][3];
    for (int a = 0; a < 2; ++a) {
        Eval deltay = Eval(qj.p[a].v) - qi.p[a];  // i is the focus
        for (int d = 0; d < dim; ++d) { double t = xj[d] - xi[d]; grad[a][d] = deltay * (t / distSq); }
    }
    // gravity correction
    double distIn[3], distEx[3], distTot[3];
    for (int d = 0; d < 3; ++d) { distIn[d] = xi[d] - xf[d]; distEx[d] = xj[d] - xf[d]; distTot[d] = xj[d] - xi[d]; }
    double absDistTotSq = 0.0;
    for (int d = 0; d < dim; ++d) absDistTotSq += distTot[d] * distTot[d];
    double gIn = 0.0, gEx = 0.0;
    for (int d = 0; d < dim; ++d) { gIn += C.gravity(d) * distIn[d]; gEx += C.gravity(d) * distEx[d]; }
    for (int a = 0; a < 2; ++a) {
        Eval pStatIn = -qi.rho[a] * gIn;           // focus: carries rho derivatives
        Eval pStatEx = Eval(-(qj.rho[a].v * gEx));  // exterior: value only
        Eval q = (pStatEx - pStatIn) / absDistTotSq;
        for (int d = 0; d < dim; ++d) grad[a][d] += distTot[d] * q;
        for (int d = 0; d < dim; ++d)
            if (!std::isfinite(grad[a][d].v)) throw std::runtime_error("Non-finite potential gradient");
    }
    // face permeability: entry-wise harmonic mean of isotropic tensors
    double Kf[3][3];
    for (int r = 0; r < dim; ++r)
        for (int s = 0; s < dim; ++s)
            Kf[r][s] = harmonicMean(r == s ? qi.K : 0.0, r == s ? qj.K : 0.0);
    for (int a = 0; a < 2; ++a) {
        Eval tmp(0.0);
        for (int d = 0; d < dim; ++d) tmp += grad[a][d] * nrm[d];
        bool upIsExterior = tmp.v > 0;
        Eval mob = upIsExterior ? Eval(qj.mob[a].v) : qi.mob[a];
        // filter velocity v = -mob * K grad; volume flux = v . n
        Eval vel[3];
        for (int r = 0; r < dim; ++r) {
            Eval s(0.0);
            for (int c2 = 0; c2 < dim; ++c2) s += Kf[r][c2] * grad[a][c2];
            vel[r] = s * (-mob);
        }
        Eval volFlux(0.0);
        for (int d = 0; d < dim; ++d) volFlux += vel[d] * nrm[d];
        Eval rho = upIsExterior ? Eval(qj.rho[a].v) : qi.rho[a];
        flux[a] = volFlux * rho;
    }
}

// LensProblem::boundary + ImmiscibleBoundaryRateVector, returned as a mass rate per area
// (positive = leaving through the face). kind: 0 no-flow, 1 free-flow, 2 inlet.
static void boundaryRate(const Ctx& C, int64_t ci, const Face& f, const IQ& qi, Eval rate[2],
                         int* kind) {
    double xf[3], xi[3];
    C.faceCenter(ci, f.axis, f.side, xf);
    C.center(ci, xi);
    const ewg_problem& P = C.prob;
    const int dim = C.dim;
    double xmin = 0.0, xmax = C.L[0], ymax = C.L[1], ymin = 0.0;
    bool left = xf[0] < xmin + P.eps, right = xf[0] > xmax - P.eps;
    rate[0] = Eval(0.0); rate[1] = Eval(0.0);
    if (left || right) {
        *kind = 1;
        double densityW = P.rho_w, densityN = P.rho_n;
        double pw, Sw = 1.0;
        double depth = ymax - xf[1];
        if (left) {
            double alpha = P.left_pressure_scale;
            pw = P.p_ref - alpha * densityW * C.gravity(1) * depth;
        } else {
            pw = P.p_ref - densityW * C.gravity(1) * depth;
        }
        (void)ymin;
        const Law& Lf = C.law[C.isInLens(xf) ? 1 : 0];
        double pC[2];
        capillaryPressures(pC, Lf, Sw);
        double pB[2] = {pw, pw + pC[1] - pC[0]};
        double rhoB[2] = {densityW, densityN};
        double muB[2] = {P.mu_w, P.mu_n};
        // boundary gradient (fvbasegradientcalculator.hh:277-312), i is the focus
        double distSq = 0.0;
        for (int d = 0; d < dim; ++d) { double t = xf[d] - xi[d]; distSq += t * t; }
        Eval grad[2][3];
        for (int a = 0; a < 2; ++a) {
            Eval deltay = Eval(pB[a]) - qi.p[a];
            for (int d = 0; d < dim; ++d) { double t = xf[d] - xi[d]; grad[a][d] = deltay * (t / distSq); }
        }
        double distIn[3];
        for (int d = 0; d < 3; ++d) distIn[d] = xi[d] - xf[d];
        double absDistSq = 0.0, gTimesDist = 0.0;
        for (int d = 0; d < dim; ++d) { absDistSq += distIn[d] * distIn[d]; gTimesDist += C.gravity(d) * distIn[d]; }
        for (int a = 0; a < 2; ++a) {
            Eval rhoIn = qi.rho[a];
            Eval pStatIn = -gTimesDist * rhoIn;
            Eval q = pStatIn / absDistSq;
            for (int d = 0; d < dim; ++d) grad[a][d] += distIn[d] * q;
            for (int d = 0; d < dim; ++d)
                if (!std::isfinite(grad[a][d].v)) throw std::runtime_error("Non finite potential gradient");
        }
        double nrm[3] = {0, 0, 0};
        nrm[f.axis] = f.side == 0 ? -1.0 : 1.0;
        const Law& Li = C.law[C.inLens[ci]];
        double krB[2];
        relativePermeabilities(krB, Li, Sw);
        for (int a = 0; a < 2; ++a) {
            Eval tmp(0.0);
            for (int d = 0; d < dim; ++d) tmp += grad[a][d] * nrm[d];
            Eval mob = (tmp.v > 0) ? Eval(krB[a] / muB[a]) : qi.mob[a];
            Eval volFlux(0.0);
            for (int d = 0; d < dim; ++d) {
                Eval s(0.0);
                for (int c2 = 0; c2 < dim; ++c2) s += (d == c2 ? qi.K : 0.0) * grad[a][c2];
                Eval v = s * (-mob);
                volFlux += v * nrm[d];
            }
            Eval density = (pB[a] > qi.p[a].v) ? Eval(rhoB[a]) : qi.rho[a];
            rate[a] = rate[a] + volFlux * density;
        }
        return;
    }
    bool upper = xf[1] > ymax - P.eps;
    bool inlet = upper && xf[0] > P.inlet_x_lo && xf[0] < P.inlet_x_hi;
    if (inlet && dim == 3) inlet = xf[2] > P.inlet_z_lo && xf[2] < P.inlet_z_hi;
    if (inlet) {
        *kind = 2;
        rate[1] = Eval(P.inlet_rate);
        return;
    }
    *kind = 0;
}

// FvBaseAdLocalLinearizer::linearize + FvBaseLocalResidual::eval for one element, then the
// column scatter of FvBaseLinearizer::linearizeElement_.
// FvBaseLocalResidual::eval for one element whose own DOF has the intensive quantities qi:
// fluxes, volume terms, boundary, volumetric division. `stashed` marks a finite-difference
// evaluation at deflected primary variables, which reads the storage cache and never writes it
// (fvbaselocalresidual.hh:541-567, haveStashedIntensiveQuantities()).
static void evalLocal(Ctx& C, int64_t e, const IQ& qi, double dt, int newtonIteration, bool stashed,
                      const Face f[6], int nf, const int faceDof[6], int ndof, Eval R[7][2]) {
    for (int d = 0; d < ndof; ++d) { R[d][0] = Eval(0.0); R[d][1] = Eval(0.0); }
    // evalFluxes: residual[i] += flux, residual[j] -= flux
    for (int k = 0; k < nf; ++k) {
        if (f[k].nbr < 0) continue;
        Eval flux[2];
        interiorFlux(C, e, f[k].nbr, f[k], qi, C.iqCache[f[k].nbr], flux);
        double alpha = 1.0;  // extrusion factor
        alpha *= C.area(f[k].axis);
        for (int a = 0; a < 2; ++a) flux[a] = flux[a] * alpha;
        int j = faceDof[k];
        for (int a = 0; a < 2; ++a) { R[0][a] += flux[a]; R[j][a] -= flux[a]; }
    }
    // evalVolumeTerms_ (focus DOF only; numPrimaryDof == 1)
    {
        double V = C.vol() * 1.0;
        Eval tmp[2];
        storageOf<Eval>(qi, tmp);
        double tmp2[2];
        if (newtonIteration == 0 && !stashed) {
            if (!C.recycleStorage) {
                IQ qold = computeIQ(C, e, C.sol[1].data(), false);
                storageOf<double>(qold, tmp2);
            } else {
                tmp2[0] = tmp[0].v; tmp2[1] = tmp[1].v;
            }
            C.storageOld[2 * e] = tmp2[0]; C.storageOld[2 * e + 1] = tmp2[1];
        } else {
            tmp2[0] = C.storageOld[2 * e]; tmp2[1] = C.storageOld[2 * e + 1];
        }
        for (int a = 0; a < 2; ++a) {
            tmp[a] -= Eval(tmp2[a]);
            tmp[a] *= Eval(V / dt);
            R[0][a] += tmp[a];
        }
        // source term: LensProblem::source is zero
        for (int a = 0; a < 2; ++a) { Eval src(0.0); src = src * V; R[0][a] -= src; }
    }
    // evalBoundary_
    for (int k = 0; k < nf; ++k) {
        if (f[k].nbr >= 0) continue;
        Eval rate[2]; int kind;
        boundaryRate(C, e, f[k], qi, rate, &kind);
        for (int a = 0; a < 2; ++a) { rate[a] = rate[a] * (C.area(f[k].axis) * 1.0); R[0][a] += rate[a]; }
    }
    // volumetric residual
    for (int d = 0; d < ndof; ++d) {
        double V = C.vol();
        for (int a = 0; a < 2; ++a) R[d][a] /= V;
    }
}

// FvBaseAdLocalLinearizer::linearize (AD) or FvBaseFdLocalLinearizer::linearize (finite
// differences, fvbasefdlocallinearizer.hh:221-237, 393-453) for one element, then the column
// scatter of FvBaseLinearizer::linearizeElement_.
static void linearizeElement(Ctx& C, int64_t e, double dt, int newtonIteration,
                             const std::vector<int32_t>& diagPos, double* errOut) {
    Face f[6];
    C.faces(e, f);
    const int nf = C.numFaces();
    // stencil DOFs: the element, then one DOF per neighbouring element (intersection order)
    int64_t dofs[7]; int ndof = 0;
    dofs[ndof++] = e;
    int faceDof[6];
    for (int k = 0; k < nf; ++k) { faceDof[k] = -1; if (f[k].nbr >= 0) { faceDof[k] = ndof; dofs[ndof++] = f[k].nbr; } }
    // local residual: one 2-vector of AD values per stencil DOF (eq index == phase index)
    Eval R[7][2];
    evalLocal(C, e, C.iqCache[e], dt, newtonIteration, false, f, nf, faceDof, ndof, R);
    if (C.fd) {
        // BaseEpsilon / primaryVarWeight; the weight is 10 / p_ref for the pressure, 1 otherwise
        const double baseEps = std::max(0.9123e-10, std::numeric_limits<double>::epsilon() * 1.23e3);
        for (int pv = 0; pv < 2; ++pv) {
            const double pvWeight = pv == 0 ? 10 / C.refPressure : 1.0;
            const double eps = baseEps / pvWeight;
            double priVars[2] = {C.sol[0][2 * e], C.sol[0][2 * e + 1]};
            double delta = 0.0;
            double deriv[7][2];
            Eval Rp[7][2];
            if (C.fdMethod >= 0) {
                priVars[pv] += eps;
                delta += eps;
                evalLocal(C, e, computeIQAt(C, e, priVars[0], priVars[1], false), dt, newtonIteration, true, f, nf, faceDof, ndof, Rp);
                for (int d = 0; d < ndof; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] = Rp[d][a].v;
            } else {
                for (int d = 0; d < ndof; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] = R[d][a].v;
            }
            if (C.fdMethod <= 0) {
                priVars[pv] -= delta + eps;
                delta += eps;
                evalLocal(C, e, computeIQAt(C, e, priVars[0], priVars[1], false), dt, newtonIteration, true, f, nf, faceDof, ndof, Rp);
                for (int d = 0; d < ndof; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] -= Rp[d][a].v;
            } else {
                for (int d = 0; d < ndof; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] -= R[d][a].v;
            }
            for (int d = 0; d < ndof; ++d) for (int a = 0; a < 2; ++a) R[d][a].d[pv] = deriv[d][a] / delta;
        }
    }
    // scatter: residual row of the focus DOF and the Jacobian column of the focus DOF
    C.resid[2 * e] = R[0][0].v; C.resid[2 * e + 1] = R[0][1].v;
    double err = std::max(std::abs(R[0][0].v), std::abs(R[0][1].v));
    if (!std::isfinite(R[0][0].v) || !std::isfinite(R[0][1].v)) err = std::numeric_limits<double>::infinity();
    *errOut = std::max(*errOut, err);
    for (int d = 0; d < ndof; ++d) {
        int64_t row = dofs[d];
        // locate block (row, e)
        int32_t pos = -1;
        if (row == e) pos = diagPos[e];
        else {
            for (int32_t q = C.rowPtr[row]; q < C.rowPtr[row + 1]; ++q) if (C.colIdx[q] == e) { pos = q; break; }
        }
        double* B = &C.blocks[4 * (size_t)pos];
        for (int eq = 0; eq < 2; ++eq)
            for (int pv = 0; pv < 2; ++pv) B[2 * eq + pv] = R[d][eq].d[pv];
    }
}

static void parallelFor(int nthreads, int64_t n, const std::function<void(int64_t, int64_t, int)>& fn) {
    if (nthreads <= 1 || n < 4096) { fn(0, n, 0); return; }
    std::vector<std::thread> th;
    int64_t chunk = (n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; ++t) {
        int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
        if (b >= e) break;
        th.emplace_back(fn, b, e, t);
    }
    for (auto& t : th) t.join();
}

static void buildPattern(Ctx& C) {
    // createMatrix_: row i holds {i} and its face neighbours, columns sorted (std::set)
    C.rowPtr.assign(C.N + 1, 0);
    std::vector<int32_t> cols;
    cols.reserve((size_t)C.N * (2 * C.dim + 1));
    Face f[6];
    for (int64_t c = 0; c < C.N; ++c) {
        std::set<int64_t> s;
        s.insert(c);
        C.faces(c, f);
        for (int k = 0; k < C.numFaces(); ++k) if (f[k].nbr >= 0) s.insert(f[k].nbr);
        for (int64_t v : s) cols.push_back((int32_t)v);
        C.rowPtr[c + 1] = (int32_t)cols.size();
    }
    C.colIdx = std::move(cols);
    C.blocks.assign(C.colIdx.size() * 4, 0.0);
}

static std::vector<int32_t> diagPositions(const Ctx& C) {
    std::vector<int32_t> d(C.N);
    for (int64_t r = 0; r < C.N; ++r)
        for (int32_t q = C.rowPtr[r]; q < C.rowPtr[r + 1]; ++q) if (C.colIdx[q] == r) { d[r] = q; break; }
    return d;
}

static double linearize(Ctx& C, double dt, int newtonIteration) {
    // resetSystem_
    std::fill(C.resid.begin(), C.resid.end(), 0.0);
    std::fill(C.blocks.begin(), C.blocks.end(), 0.0);
    std::vector<int32_t> diag = diagPositions(C);
    // intensive-quantity cache (EnableIntensiveQuantityCache): one evaluation per DOF
    C.iqCache.resize(C.N);
    const double* x = C.sol[0].data();
    parallelFor(C.nthreads, C.N, [&](int64_t b, int64_t e, int) {
        for (int64_t c = b; c < e; ++c) C.iqCache[c] = computeIQ(C, c, x, true);
    });
    std::vector<double> errs(std::max(1, C.nthreads), 0.0);
    std::vector<std::string> exc(std::max(1, C.nthreads));
    parallelFor(C.nthreads, C.N, [&](int64_t b, int64_t e, int t) {
        try {
            for (int64_t c = b; c < e; ++c) linearizeElement(C, c, dt, newtonIteration, diag, &errs[t]);
        } catch (const std::exception& ex) { exc[t] = ex.what(); }
    });
    for (auto& s : exc) if (!s.empty()) throw std::runtime_error(s);
    double err = 0.0;
    for (double v : errs) err = std::max(err, v);
    return err;
}

// ---------------------------------------------------------------------------------------------
// 2x2 block helpers (row-major [eq][pv])
static inline void inv2(const double* A, double* out) {
    double det = A[0] * A[3] - A[1] * A[2];
    if (det == 0.0 || !std::isfinite(det)) throw std::runtime_error("singular diagonal block");
    double di = 1.0 / det;
    out[0] = A[3] * di; out[1] = -A[1] * di; out[2] = -A[2] * di; out[3] = A[0] * di;
}
static inline void mul2(const double* A, const double* B, double* out) {
    double o[4];
    o[0] = A[0] * B[0] + A[1] * B[2]; o[1] = A[0] * B[1] + A[1] * B[3];
    o[2] = A[2] * B[0] + A[3] * B[2]; o[3] = A[2] * B[1] + A[3] * B[3];
    std::memcpy(out, o, sizeof(o));
}
static inline void mmv2(const double* A, const double* x, double* y) {  // y -= A x
    y[0] -= A[0] * x[0]; y[0] -= A[1] * x[1];
    y[1] -= A[2] * x[0]; y[1] -= A[3] * x[1];
}

// A block-sparse matrix in BCRS with sorted columns (a dune BCRSMatrix<FieldMatrix<double,2,2>>).
struct Bcrs {
    int64_t n = 0;
    std::vector<int32_t> rp, ci;
    std::vector<double> v;
    std::vector<int32_t> diag;
    void findDiag() {
        diag.assign(n, -1);
        for (int64_t r = 0; r < n; ++r)
            for (int32_t q = rp[r]; q < rp[r + 1]; ++q) if (ci[q] == r) diag[r] = q;
    }
    void mv(const double* x, double* y) const {
        for (int64_t r = 0; r < n; ++r) {
            double a0 = 0.0, a1 = 0.0;
            for (int32_t q = rp[r]; q < rp[r + 1]; ++q) {
                const double* B = &v[4 * (size_t)q]; const double* xx = &x[2 * (size_t)ci[q]];
                a0 += B[0] * xx[0]; a0 += B[1] * xx[1];
                a1 += B[2] * xx[0]; a1 += B[3] * xx[1];
            }
            y[2 * r] = a0; y[2 * r + 1] = a1;
        }
    }
};

// dune-istl bilu0_decomposition: left-looking, stored inverse diagonal
static void bilu0(Bcrs& A) {
    for (int64_t i = 0; i < A.n; ++i) {
        int32_t ij = A.rp[i];
        for (; ij < A.rp[i + 1] && A.ci[ij] < i; ++ij) {
            int32_t j = A.ci[ij];
            int32_t jj = A.diag[j];
            double* Lij = &A.v[4 * (size_t)ij];
            mul2(Lij, &A.v[4 * (size_t)jj], Lij);  // A_ij * inv(A_jj)
            int32_t jk = jj + 1, ik = ij + 1;
            while (ik < A.rp[i + 1] && jk < A.rp[j + 1]) {
                if (A.ci[ik] == A.ci[jk]) {
                    double B[4];
                    mul2(Lij, &A.v[4 * (size_t)jk], B);
                    double* Aik = &A.v[4 * (size_t)ik];
                    for (int t = 0; t < 4; ++t) Aik[t] -= B[t];
                    ++ik; ++jk;
                } else if (A.ci[ik] < A.ci[jk]) ++ik; else ++jk;
            }
        }
        if (ij >= A.rp[i + 1] || A.ci[ij] != i) throw std::runtime_error("diagonal entry missing");
        double inv[4];
        inv2(&A.v[4 * (size_t)ij], inv);
        std::memcpy(&A.v[4 * (size_t)ij], inv, sizeof(inv));
    }
}
// dune-istl bilu_backsolve
static void biluApply(const Bcrs& A, const double* d, double* v) {
    for (int64_t i = 0; i < A.n; ++i) {
        double rhs[2] = {d[2 * i], d[2 * i + 1]};
        for (int32_t q = A.rp[i]; q < A.rp[i + 1] && A.ci[q] < i; ++q) mmv2(&A.v[4 * (size_t)q], &v[2 * (size_t)A.ci[q]], rhs);
        v[2 * i] = rhs[0]; v[2 * i + 1] = rhs[1];
    }
    for (int64_t i = A.n - 1; i >= 0; --i) {
        double rhs[2] = {v[2 * i], v[2 * i + 1]};
        int32_t q = A.rp[i + 1] - 1;
        for (; A.ci[q] > i; --q) mmv2(&A.v[4 * (size_t)q], &v[2 * (size_t)A.ci[q]], rhs);
        const double* D = &A.v[4 * (size_t)q];
        v[2 * i] = D[0] * rhs[0] + D[1] * rhs[1];
        v[2 * i + 1] = D[2] * rhs[0] + D[3] * rhs[1];
    }
}

struct Precond {
    int kind = EWG_PRECOND_ILU0;
    int ordering = ORC_ORDER_NATURAL;
    double w = 1.0;
    Bcrs F;                         // factor (ILU) in the chosen ordering
    std::vector<int64_t> perm, iperm;  // new index -> old, old -> new
    std::vector<int8_t> colourOf;      // ORC_ORDER_COLOURS: colour of each row
    std::vector<double> Dinv;        // Jacobi
    std::vector<double> tin, tout;
    void setup(const Ctx& C, const Bcrs& A) {
        if (kind == EWG_PRECOND_JACOBI) {
            Dinv.assign(4 * (size_t)A.n, 0.0);
            for (int64_t i = 0; i < A.n; ++i) inv2(&A.v[4 * (size_t)A.diag[i]], &Dinv[4 * (size_t)i]);
            return;
        }
        perm.resize(A.n); iperm.resize(A.n);
        if (ordering == ORC_ORDER_NATURAL) {
            for (int64_t i = 0; i < A.n; ++i) perm[i] = iperm[i] = i;
        } else if (ordering == ORC_ORDER_COLOURS) {
            int64_t k = 0;
            for (int color = 0; color < 8; ++color)
                for (int64_t c = 0; c < A.n; ++c)
                    if (colourOf[c] == color) { perm[k] = c; iperm[c] = k; ++k; }
        } else if (ordering == ORC_ORDER_BOX8) {
            // 2x2x2 boxes in eight colours: a cell's colour is bit 1 of (i, j, k), its place in
            // its box bit 0; colour-major, then box (i/4, j/4, k/4) in natural order, then the
            // cell's place in the box (x fastest). Boxes of one colour are never adjacent.
            std::vector<std::array<int64_t, 4>> key((size_t)A.n);
            const int64_t nbx = (C.n[0] + 3) / 4, nby = (C.n[1] + 3) / 4;
            for (int64_t c = 0; c < A.n; ++c) {
                int64_t i, j, kk; C.ijk(c, i, j, kk);
                const int64_t colour = ((i >> 1) & 1) | (((j >> 1) & 1) << 1) | (((kk >> 1) & 1) << 2);
                const int64_t box = (i >> 2) + nbx * ((j >> 2) + nby * (kk >> 2));
                const int64_t q = (i & 1) | ((j & 1) << 1) | ((kk & 1) << 2);
                key[(size_t)c] = {colour, box, q, c};
            }
            for (int64_t c = 0; c < A.n; ++c) perm[c] = c;
            std::sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return key[(size_t)a] < key[(size_t)b]; });
            for (int64_t k = 0; k < A.n; ++k) iperm[perm[k]] = k;
        } else {
            int64_t k = 0;
            for (int color = 0; color < 2; ++color)
                for (int64_t c = 0; c < A.n; ++c) {
                    int64_t i, j, kk; C.ijk(c, i, j, kk);
                    if (((i + j + kk) & 1) == color) { perm[k] = c; iperm[c] = k; ++k; }
                }
        }
        F.n = A.n; F.rp.assign(A.n + 1, 0); F.ci.clear(); F.v.clear();
        for (int64_t r = 0; r < A.n; ++r) {
            int64_t o = perm[r];
            std::vector<std::pair<int32_t, int32_t>> row;
            for (int32_t q = A.rp[o]; q < A.rp[o + 1]; ++q) row.push_back({(int32_t)iperm[A.ci[q]], q});
            std::sort(row.begin(), row.end());
            for (auto& pr : row) {
                F.ci.push_back(pr.first);
                for (int t = 0; t < 4; ++t) F.v.push_back(A.v[4 * (size_t)pr.second + t]);
            }
            F.rp[r + 1] = (int32_t)F.ci.size();
        }
        F.findDiag();
        bilu0(F);
        tin.resize(2 * A.n); tout.resize(2 * A.n);
    }
    void apply(const double* d, double* v) {
        if (kind == EWG_PRECOND_JACOBI) {
            for (int64_t i = 0; i < (int64_t)(Dinv.size() / 4); ++i) {
                const double* D = &Dinv[4 * (size_t)i];
                v[2 * i] = w * (D[0] * d[2 * i] + D[1] * d[2 * i + 1]);
                v[2 * i + 1] = w * (D[2] * d[2 * i] + D[3] * d[2 * i + 1]);
            }
            return;
        }
        for (int64_t r = 0; r < F.n; ++r) { tin[2 * r] = d[2 * perm[r]]; tin[2 * r + 1] = d[2 * perm[r] + 1]; }
        biluApply(F, tin.data(), tout.data());
        for (int64_t r = 0; r < F.n; ++r) { v[2 * perm[r]] = w * tout[2 * r]; v[2 * perm[r] + 1] = w * tout[2 * r + 1]; }
    }
};

struct BreakdownError : std::runtime_error { using std::runtime_error::runtime_error; };

// CombinedCriterion (combinedcriterion.hh:112-205)
struct Criterion {
    double relTol, absTol, maxRes;
    double resErr = 0, lastResErr = 0, initResErr = 0;
    bool stagnates = false;
    void updateErrors(const double* change, const double* resid, int64_t n2) {
        lastResErr = resErr;
        resErr = 0.0;
        stagnates = true;
        for (int64_t i = 0; i < n2; ++i) {
            resErr = std::max(resErr, std::abs(resid[i]));
            if (stagnates && change[i] != 0.0) stagnates = false;
        }
    }
    void setInitial(const double* x, const double* r, int64_t n2) {
        updateErrors(x, r, n2);
        stagnates = false;
        resErr = std::max(resErr, std::numeric_limits<double>::min() * 1e10);
        initResErr = resErr; lastResErr = resErr;
    }
    double reduction() const { return resErr / std::max(1e-20, initResErr); }
    bool converged() const { return reduction() <= relTol || resErr <= absTol; }
    bool failed() const { return !converged() && (stagnates || resErr > maxRes); }
};

static double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// BiCGStabSolver::apply (bicgstabsolver.hh:116-326), including its aliasing (h == x, s == r,
// t == y) and the criterion update order.
// Extension (off = exactly the reference): when the shadow residual has become orthogonal to
// the residual (|r0hat . r| <= 1e-12 |r0hat| |r|), restart with r0hat = r, keeping x.
// Second extension (off = exactly the reference): on convergence the true residual b - A x is
// recomputed; if it misses the criterion by more than a factor 10 (the recursively updated
// residual has drifted), the iteration continues from x with r = r0hat = b - A x (at most 3 times).
static bool bicgstab(const Bcrs& A, Precond& M, const std::vector<double>& b, std::vector<double>& x,
                     Criterion& crit, int maxIter, bool restartOnBreakdown, bool verifyTrue,
                     int* iters, int* restarts) {
    const double breakdownEps = std::numeric_limits<double>::min() * 1e10;
    const int64_t n2 = (int64_t)b.size();
    x.assign(n2, 0.0);
    std::vector<double> r = b;
    crit.setInitial(x.data(), r.data(), n2);
    *iters = 0;
    *restarts = 0;
    if (crit.converged()) return true;
    std::vector<double> r0hat = b;
    double r0r0 = dot(r0hat, r0hat);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    std::vector<double> v(n2, 0.0), p(n2, 0.0), y(n2, 0.0), z(n2, 0.0);
    std::vector<double>& h = x; std::vector<double>& s = r; std::vector<double>& t = y;
    int replacements = 0;
    // true-residual check; returns true when the iteration must go on from the replaced residual
    auto replaceResidual = [&]() -> bool {
        if (!verifyTrue || replacements >= 3) return false;
        std::vector<double> ax(n2);
        A.mv(x.data(), ax.data());
        double err = 0.0;
        for (int64_t i = 0; i < n2; ++i) { r[i] = b[i] - ax[i]; err = std::max(err, std::abs(r[i])); }
        if (err / std::max(1e-20, crit.initResErr) <= 10 * crit.relTol || err <= 10 * crit.absTol) return false;
        ++replacements;
        ++*restarts;
        r0hat = r; r0r0 = dot(r, r);
        rho = 1.0; alpha = 1.0; omega = 1.0;
        std::fill(v.begin(), v.end(), 0.0); std::fill(p.begin(), p.end(), 0.0);
        crit.lastResErr = crit.resErr; crit.resErr = err; crit.stagnates = false;
        return true;
    };
    int it = 0;
    for (; it < maxIter; ++it) {
        double rho_i = dot(r0hat, r);
        if (restartOnBreakdown) {
            double rr = dot(r, r);
            if (std::abs(rho_i) <= 1e-12 * std::sqrt(r0r0) * std::sqrt(rr)) {
                r0hat = r; r0r0 = rr; rho_i = rr;
                rho = 1.0; alpha = 1.0; omega = 1.0;
                std::fill(v.begin(), v.end(), 0.0); std::fill(p.begin(), p.end(), 0.0);
                ++*restarts;
            }
        }
        if (std::abs(rho) <= breakdownEps || std::abs(omega) <= breakdownEps)
            throw BreakdownError("Breakdown of the BiCGStab solver (division by zero)");
        double beta = (rho_i / rho) * (alpha / omega);
        rho = rho_i;
        for (int64_t i = 0; i < n2; ++i) {
            double tmp = v[i];
            tmp *= omega; tmp -= p[i]; tmp *= -beta;
            p[i] = r[i]; p[i] += tmp;
        }
        M.apply(p.data(), y.data());
        A.mv(y.data(), v.data());
        double denom = dot(r0hat, v);
        if (std::abs(denom) <= breakdownEps) throw BreakdownError("Breakdown of the BiCGStab solver (division by zero)");
        alpha = rho_i / denom;
        if (std::abs(alpha) <= breakdownEps) throw BreakdownError("Breakdown of the BiCGStab solver (stagnation detected)");
        for (int64_t i = 0; i < n2; ++i) {
            double tmp = y[i]; tmp *= alpha; tmp += x[i]; h[i] = tmp;
            tmp = v[i]; tmp *= alpha; s[i] -= tmp;
        }
        crit.updateErrors(y.data(), s.data(), n2);
        if (crit.converged()) {
            if (!replaceResidual()) { *iters = it; return true; }
            continue;
        }
        if (crit.failed()) { *iters = it; return false; }
        z = s;
        M.apply(s.data(), z.data());
        A.mv(z.data(), t.data());
        denom = dot(t, t);
        if (std::abs(denom) <= breakdownEps) throw BreakdownError("Breakdown of the BiCGStab solver (division by zero)");
        omega = dot(t, s) / denom;
        if (std::abs(omega) <= breakdownEps) throw BreakdownError("Breakdown of the BiCGStab solver (stagnation detected)");
        for (int64_t i = 0; i < n2; ++i) x[i] += omega * z[i];
        crit.updateErrors(z.data(), r.data(), n2);
        if (crit.converged()) {
            if (!replaceResidual()) { *iters = it; return true; }
            continue;
        }
        if (crit.failed()) { *iters = it; return false; }
        for (int64_t i = 0; i < n2; ++i) r[i] += -omega * t[i];
    }
    *iters = it;
    return false;
}

static Bcrs systemMatrix(const Ctx& C) {
    Bcrs A; A.n = C.N; A.rp = C.rowPtr; A.ci = C.colIdx; A.v = C.blocks; A.findDiag();
    return A;
}

// ---------------------------------------------------------------------------------------------
// Vertex-centred finite volumes (VcfvDiscretization, discretizations/vcfv/) for the same model and
// problem with P1 finite-element gradients (UseP1FiniteElementGradients, as lens_immiscible_vcfv_ad
// sets): DOFs at the grid vertices, control volumes from the sub-control volumes (SCVs) that each
// element gives its corners, fluxes over the sub-control-volume faces (SCVFs) that join the element
// centre to its edges (vcfvstencil.hh:866-1016). Structured grids of axis-aligned boxes: every
// element has the same local geometry, built once from the reference element in DUNE's numbering
// (vertex v has local coordinates given by its bits; edges and faces as in the tables of
// vcfvstencil.hh:595-716), with global vectors taken relative to the element's lower corner.

struct VGeom {
    int dim = 2, nv = 4, ne = 4, nf = 4, nfv = 2;
    double h[3] = {1, 1, 1};
    int vb[8][3] = {};
    int ei[12] = {}, ej[12] = {};        // SCVF interior / exterior vertex
    double ip[12][3] = {};               // SCVF integration point (local)
    double nrm[12][3] = {}, area[12] = {};
    double G[12][8][3] = {};             // global P1 shape-function gradients at ip
    double scvVol = 0.0;
    double scvCenter[8][3] = {};         // local
    int fv[6][4] = {};                   // vertices of each element face
    double bip[6][4][3] = {}, barea[6][4] = {};
    double fnrm[6][3] = {};              // outer unit normal of each element face
    int faxis[6] = {}, fside[6] = {};
};

static void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// normalOfQuadrilateral3D (vcfvstencil.hh:568-583): 0.5 (p2 - p0) x (p3 - p1)
static void quadNormal(const double p0[3], const double p1[3], const double p2[3], const double p3[3], double n[3]) {
    double a[3], b[3];
    for (int d = 0; d < 3; ++d) { a[d] = p2[d] - p0[d]; b[d] = p3[d] - p1[d]; }
    cross3(a, b, n);
    for (int d = 0; d < 3; ++d) n[d] *= 0.5;
}
static double norm3(const double n[3], int dim) {
    double s = 0.0;
    for (int d = 0; d < dim; ++d) s += n[d] * n[d];
    return std::sqrt(s);
}

static VGeom makeVGeom(int dim, const double h[3]) {
    VGeom g;
    g.dim = dim;
    g.nv = 1 << dim;
    g.ne = dim == 2 ? 4 : 12;
    g.nf = 2 * dim;
    g.nfv = dim == 2 ? 2 : 4;
    for (int d = 0; d < 3; ++d) g.h[d] = d < dim ? h[d] : 1.0;
    for (int v = 0; v < g.nv; ++v)
        for (int d = 0; d < 3; ++d) g.vb[v][d] = d < dim ? (v >> d) & 1 : 0;
    auto glob = [&](const double l[3], double o[3]) { for (int d = 0; d < 3; ++d) o[d] = d < dim ? l[d] * g.h[d] : 0.0; };
    double elemL[3] = {0.5, 0.5, dim == 3 ? 0.5 : 0.0}, elemG[3];
    glob(elemL, elemG);
    // element faces: 2a + s is the face with x_a = s (YaspGrid intersection order)
    double faceL[6][3];
    for (int f = 0; f < g.nf; ++f) {
        int a = f >> 1, sd = f & 1;
        g.faxis[f] = a; g.fside[f] = sd;
        for (int d = 0; d < 3; ++d) faceL[f][d] = d < dim ? 0.5 : 0.0;
        faceL[f][a] = sd;
        for (int d = 0; d < 3; ++d) g.fnrm[f][d] = 0.0;
        g.fnrm[f][a] = sd ? 1.0 : -1.0;
        int m = 0;
        for (int v = 0; v < g.nv; ++v) if (g.vb[v][a] == sd) g.fv[f][m++] = v;
    }
    // edges (reference-element numbering)
    static const int e2[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};
    static const int e3[12][2] = {{0, 4}, {1, 5}, {2, 6}, {3, 7}, {0, 2}, {1, 3},
                                  {0, 1}, {2, 3}, {4, 6}, {5, 7}, {4, 5}, {6, 7}};
    static const unsigned edgeToFaceHex[2][12] = {{0, 2, 3, 1, 4, 1, 2, 4, 0, 5, 5, 3},
                                                  {2, 1, 0, 3, 0, 4, 4, 3, 5, 1, 2, 5}};
    double edgeL[12][3], edgeG[12][3], faceG[6][3];
    for (int f = 0; f < g.nf; ++f) glob(faceL[f], faceG[f]);
    for (int k = 0; k < g.ne; ++k) {
        int a = dim == 2 ? e2[k][0] : e3[k][0], b = dim == 2 ? e2[k][1] : e3[k][1];
        for (int d = 0; d < 3; ++d) edgeL[k][d] = d < dim ? 0.5 * (g.vb[a][d] + g.vb[b][d]) : 0.0;
        glob(edgeL[k], edgeG[k]);
        int i = a, j = b;
        if (g.ne == 4 && (i == 2 || j == 2)) std::swap(i, j);
        g.ei[k] = i; g.ej[k] = j;
        double n[3] = {0, 0, 0};
        if (dim == 2) {
            for (int d = 0; d < 3; ++d) g.ip[k][d] = (edgeL[k][d] + elemL[d]) * 0.5;
            double diff[3];
            for (int d = 0; d < 2; ++d) diff[d] = elemG[d] - edgeG[k][d];
            n[0] = diff[1]; n[1] = -diff[0];
            double xi[3], xj[3], li[3], lj[3];
            for (int d = 0; d < 3; ++d) { li[d] = g.vb[i][d]; lj[d] = g.vb[j][d]; }
            glob(li, xi); glob(lj, xj);
            double dot = 0.0;
            for (int d = 0; d < 2; ++d) dot += n[d] * (xj[d] - xi[d]);
            if (dot < 0) for (int d = 0; d < 2; ++d) n[d] *= -1;
        } else {
            unsigned lf = edgeToFaceHex[0][k], rf = edgeToFaceHex[1][k];
            for (int d = 0; d < 3; ++d) g.ip[k][d] = (((edgeL[k][d] + elemL[d]) + faceL[lf][d]) + faceL[rf][d]) * 0.25;
            quadNormal(edgeG[k], faceG[rf], elemG, faceG[lf], n);
        }
        g.area[k] = norm3(n, dim);
        for (int d = 0; d < 3; ++d) g.nrm[k][d] = d < dim ? n[d] / g.area[k] : 0.0;
        // P1 (Q1) shape-function gradients at the integration point, mapped by the inverse
        // transposed Jacobian diag(1/h)
        for (int v = 0; v < g.nv; ++v)
            for (int d = 0; d < dim; ++d) {
                double q = g.vb[v][d] ? 1.0 : -1.0;
                for (int e = 0; e < dim; ++e)
                    if (e != d) q *= g.vb[v][e] ? g.ip[k][e] : 1.0 - g.ip[k][e];
                g.G[k][v][d] = (1.0 / g.h[d]) * q;
            }
    }
    // sub-control volumes: the box between the vertex and the element centre
    double vol = 1.0;
    for (int d = 0; d < dim; ++d) vol *= g.h[d];
    g.scvVol = vol / g.nv;
    for (int v = 0; v < g.nv; ++v)
        for (int d = 0; d < 3; ++d) g.scvCenter[v][d] = d < dim ? (g.vb[v][d] + elemL[d]) * 0.5 : 0.0;
    // boundary sub-faces: one per (element face, vertex of the face)
    static const int leftEdgeHex[6][8] = {{0, -1, 4, -1, 8, -1, 2, -1}, {-1, 5, -1, 3, -1, 1, -1, 9},
                                          {6, 1, -1, -1, 0, 10, -1, -1}, {-1, -1, 2, 7, -1, -1, 11, 3},
                                          {4, 6, 7, 5, -1, -1, -1, -1}, {-1, -1, -1, -1, 10, 9, 8, 11}};
    static const int rightEdgeHex[6][8] = {{4, -1, 2, -1, 0, -1, 8, -1}, {-1, 1, -1, 5, -1, 9, -1, 3},
                                           {0, 6, -1, -1, 10, 1, -1, -1}, {-1, -1, 7, 3, -1, -1, 2, 11},
                                           {6, 5, 4, 7, -1, -1, -1, -1}, {-1, -1, -1, -1, 8, 10, 11, 9}};
    for (int f = 0; f < g.nf; ++f)
        for (int m = 0; m < g.nfv; ++m) {
            int v = g.fv[f][m];
            double vl[3] = {(double)g.vb[v][0], (double)g.vb[v][1], (double)g.vb[v][2]};
            if (dim == 2) {
                for (int d = 0; d < 3; ++d) g.bip[f][m][d] = (vl[d] + faceL[f][d]) * 0.5;
                int a = g.faxis[f];
                g.barea[f][m] = 0.5 * g.h[1 - a];  // half of the face length
            } else {
                int le = leftEdgeHex[f][v], re = rightEdgeHex[f][v];
                for (int d = 0; d < 3; ++d)
                    g.bip[f][m][d] = (((vl[d] + faceL[f][d]) + edgeL[le][d]) + edgeL[re][d]) * 0.25;
                double vg[3], n[3];
                glob(vl, vg);
                quadNormal(vg, edgeG[re], faceG[f], edgeG[le], n);
                g.barea[f][m] = norm3(n, 3);
            }
        }
    return g;
}

struct VCtx {
    int dim = 2, n[3] = {1, 1, 1};   // elements per axis
    int nvx[3] = {1, 1, 1};          // vertices per axis
    double L[3] = {1, 1, 1}, h[3] = {1, 1, 1};
    int64_t NE = 0, NV = 0;
    ewg_problem prob{};
    Law law[2];
    VGeom geo;
    std::vector<double> perm;               // per vertex
    std::vector<unsigned char> inLens;      // per vertex
    std::vector<double> totVol;             // dofTotalVolume per vertex
    std::vector<double> sol[2], storageOld, resid;
    std::vector<int32_t> rowPtr, colIdx;
    std::vector<double> blocks;
    std::vector<IQ> iqCache;
    bool recycleStorage = true;
    // FiniteDifferenceLocalLinearizer with NumericDifferenceMethod fdMethod and the reference
    // pressure of ImmiscibleModel::updateBegin (p_w of the first DOF) for the pressure weight
    bool fd = false;
    int fdMethod = 1;
    double refPressure = -1.0;
    int nthreads = 1;
    std::string err;

    double gravity(int a) const { return a == 1 ? -prob.gravity : 0.0; }
    void vijk(int64_t v, int64_t id[3]) const {
        id[0] = v % nvx[0]; id[1] = (v / nvx[0]) % nvx[1]; id[2] = v / ((int64_t)nvx[0] * nvx[1]);
    }
    int64_t vindex(int64_t i, int64_t j, int64_t k) const { return i + nvx[0] * (j + (int64_t)nvx[1] * k); }
    void vpos(int64_t v, double x[3]) const {
        int64_t id[3]; vijk(v, id);
        for (int d = 0; d < 3; ++d) x[d] = d < dim ? id[d] * h[d] : 0.0;
    }
    void eijk(int64_t e, int64_t id[3]) const {
        id[0] = e % n[0]; id[1] = (e / n[0]) % n[1]; id[2] = e / ((int64_t)n[0] * n[1]);
    }
    // global vertex of local vertex lv of element e
    int64_t evert(const int64_t eid[3], int lv) const {
        return vindex(eid[0] + geo.vb[lv][0], eid[1] + geo.vb[lv][1], eid[2] + (dim == 3 ? geo.vb[lv][2] : 0));
    }
    bool isInLens(const double x[3]) const {
        for (int a = 0; a < dim; ++a)
            if (x[a] < prob.lens_lo[a] - prob.eps || x[a] > prob.lens_hi[a] + prob.eps) return false;
        return true;
    }
};

static IQ computeVIQAt(const VCtx& C, int64_t v, double pw, double sw) {
    IQ q;
    const Law& L = C.law[C.inLens[v]];
    Eval Sw = Eval::variable(sw, 1);
    q.S[0] = Sw;
    q.S[1] = 1.0 - (Eval(0.0) + Sw);
    Eval pC[2];
    capillaryPressures(pC, L, q.S[0]);
    relativePermeabilities(q.kr, L, q.S[0]);
    Eval p0 = Eval::variable(pw, 0);
    for (int a = 0; a < 2; ++a) q.p[a] = p0 + (pC[a] - pC[0]);
    q.mu[0] = Eval(C.prob.mu_w); q.mu[1] = Eval(C.prob.mu_n);
    q.rho[0] = Eval(C.prob.rho_w); q.rho[1] = Eval(C.prob.rho_n);
    for (int a = 0; a < 2; ++a) q.mob[a] = q.kr[a] / q.mu[a];
    q.porosity = C.prob.porosity;
    q.K = C.perm[v];
    return q;
}
static IQ computeVIQ(const VCtx& C, int64_t v, const double* x) { return computeVIQAt(C, v, x[2 * v], x[2 * v + 1]); }

static inline Eval focusOr(const Eval& e, bool focus) { return focus ? e : Eval(e.v); }

// Flux over SCVF k of an element whose local vertices have the intensive quantities q[],
// derivatives with respect to local vertex `focus` (darcyfluxmodule.hh:185-324 with
// P1FeGradientCalculator::calculateGradient, p1fegradientcalculator.hh:255-290; :461-527;
// immisciblelocalresidual.hh:123-149), mass per area.
static void vcfvFlux(const VCtx& C, const IQ* q[8], int k, int focus, Eval flux[2]) {
    const VGeom& g = C.geo;
    const int dim = C.dim;
    const int i = g.ei[k], j = g.ej[k];
    Eval grad[2][3];
    for (int a = 0; a < 2; ++a) {
        for (int d = 0; d < 3; ++d) grad[a][d] = Eval(0.0);
        for (int v = 0; v < g.nv; ++v) {
            Eval pv = focusOr(q[v]->p[a], v == focus);
            for (int d = 0; d < dim; ++d) grad[a][d] += pv * g.G[k][v][d];
        }
    }
    // gravity correction between the two vertices, estimated at the integration point
    double posIn[3], posEx[3], posF[3];
    for (int d = 0; d < 3; ++d) {
        posIn[d] = g.vb[i][d] * g.h[d];
        posEx[d] = g.vb[j][d] * g.h[d];
        posF[d] = g.ip[k][d] * g.h[d];
    }
    double distIn[3], distEx[3], distTot[3];
    for (int d = 0; d < 3; ++d) { distIn[d] = posIn[d] - posF[d]; distEx[d] = posEx[d] - posF[d]; distTot[d] = posEx[d] - posIn[d]; }
    double absDistTotSq = 0.0;
    for (int d = 0; d < dim; ++d) absDistTotSq += distTot[d] * distTot[d];
    double gIn = 0.0, gEx = 0.0;
    for (int d = 0; d < dim; ++d) { gIn += C.gravity(d) * distIn[d]; gEx += C.gravity(d) * distEx[d]; }
    for (int a = 0; a < 2; ++a) {
        Eval pStatIn = -(focusOr(q[i]->rho[a], i == focus) * gIn);
        Eval pStatEx = -(focusOr(q[j]->rho[a], j == focus) * gEx);
        Eval qq = (pStatEx - pStatIn) / absDistTotSq;
        for (int d = 0; d < dim; ++d) grad[a][d] += Eval(distTot[d]) * qq;
        for (int d = 0; d < dim; ++d)
            if (!std::isfinite(grad[a][d].v)) throw std::runtime_error("Non-finite potential gradient");
    }
    // intersectionIntrinsicPermeability: entry-wise harmonic mean of the two vertices' tensors
    double Kf[3][3];
    for (int r = 0; r < dim; ++r)
        for (int s2 = 0; s2 < dim; ++s2)
            Kf[r][s2] = harmonicMean(r == s2 ? q[i]->K : 0.0, r == s2 ? q[j]->K : 0.0);
    for (int a = 0; a < 2; ++a) {
        Eval tmp(0.0);
        for (int d = 0; d < dim; ++d) tmp += grad[a][d] * g.nrm[k][d];
        const int up = tmp.v > 0 ? j : i;
        Eval mob = focusOr(q[up]->mob[a], up == focus);
        Eval vel[3];
        for (int r = 0; r < dim; ++r) {
            Eval s(0.0);
            for (int c2 = 0; c2 < dim; ++c2) s += Kf[r][c2] * grad[a][c2];
            vel[r] = s * (-mob);
        }
        Eval volFlux(0.0);
        for (int d = 0; d < dim; ++d) volFlux += vel[d] * g.nrm[k][d];
        Eval rho = focusOr(q[up]->rho[a], up == focus);
        flux[a] = volFlux * rho;
    }
}

// LensProblem::boundary at boundary sub-face (f, m) of element eid, interior vertex lv: the free-flow
// state on the left / right faces with the two-point boundary gradient from the SCV centre
// (fvbasegradientcalculator.hh:277-312, darcyfluxmodule.hh:333-453), the inlet mass rate, no flow
// elsewhere; derivatives only when the vertex is the focus. Mass rate per area.
static void vcfvBoundaryRate(const VCtx& C, const int64_t eid[3], int f, int m, const IQ& qv, int lv, int64_t gv,
                             bool focus, Eval rate[2]) {
    const VGeom& g = C.geo;
    const ewg_problem& P = C.prob;
    const int dim = C.dim;
    double pos[3];  // absolute position of the integration point
    for (int d = 0; d < 3; ++d) pos[d] = d < dim ? (eid[d] + g.bip[f][m][d]) * C.h[d] : 0.0;
    double xmin = 0.0, xmax = C.L[0], ymax = C.L[1];
    bool left = pos[0] < xmin + P.eps, right = pos[0] > xmax - P.eps;
    rate[0] = Eval(0.0); rate[1] = Eval(0.0);
    if (left || right) {
        double pw, Sw = 1.0;
        double depth = ymax - pos[1];
        if (left) pw = P.p_ref - P.left_pressure_scale * P.rho_w * C.gravity(1) * depth;
        else pw = P.p_ref - P.rho_w * C.gravity(1) * depth;
        const Law& Lf = C.law[C.isInLens(pos) ? 1 : 0];
        double pC[2];
        capillaryPressures(pC, Lf, Sw);
        double pB[2] = {pw, pw + pC[1] - pC[0]};
        double rhoB[2] = {P.rho_w, P.rho_n}, muB[2] = {P.mu_w, P.mu_n};
        // relative positions: integration point, SCV centre and vertex
        double ipG[3], scvC[3], vG[3];
        for (int d = 0; d < 3; ++d) {
            ipG[d] = g.bip[f][m][d] * g.h[d];
            scvC[d] = g.scvCenter[lv][d] * g.h[d];
            vG[d] = g.vb[lv][d] * g.h[d];
        }
        double distSq = 0.0;
        for (int d = 0; d < dim; ++d) { double t = ipG[d] - scvC[d]; distSq += t * t; }
        Eval grad[2][3];
        for (int a = 0; a < 2; ++a) {
            Eval deltay = focus ? Eval(pB[a]) - qv.p[a] : Eval(pB[a] - qv.p[a].v);
            for (int d = 0; d < dim; ++d) { double t = ipG[d] - scvC[d]; grad[a][d] = deltay * (t / distSq); }
        }
        double distIn[3];
        for (int d = 0; d < 3; ++d) distIn[d] = vG[d] - ipG[d];
        double absDistSq = 0.0, gTimesDist = 0.0;
        for (int d = 0; d < dim; ++d) { absDistSq += distIn[d] * distIn[d]; gTimesDist += C.gravity(d) * distIn[d]; }
        for (int a = 0; a < 2; ++a) {
            Eval pStatIn = -gTimesDist * qv.rho[a];
            Eval qq = pStatIn / absDistSq;
            for (int d = 0; d < dim; ++d) grad[a][d] += distIn[d] * qq;
            for (int d = 0; d < dim; ++d)
                if (!std::isfinite(grad[a][d].v)) throw std::runtime_error("Non finite potential gradient");
        }
        // kr of the boundary state with the interior vertex's parameters
        const Law& Li = C.law[C.inLens[gv]];
        double krB[2];
        relativePermeabilities(krB, Li, Sw);
        for (int a = 0; a < 2; ++a) {
            Eval tmp(0.0);
            for (int d = 0; d < dim; ++d) tmp += grad[a][d] * g.fnrm[f][d];
            Eval mob = (tmp.v > 0) ? Eval(krB[a] / muB[a]) : focusOr(qv.mob[a], focus);
            Eval volFlux(0.0);
            for (int d = 0; d < dim; ++d) {
                Eval s2(0.0);
                for (int c2 = 0; c2 < dim; ++c2) s2 += (d == c2 ? qv.K : 0.0) * grad[a][c2];
                Eval vv = s2 * (-mob);
                volFlux += vv * g.fnrm[f][d];
            }
            Eval density = (pB[a] > qv.p[a].v) ? Eval(rhoB[a]) : focusOr(qv.rho[a], focus);
            rate[a] = rate[a] + volFlux * density;
        }
        return;
    }
    bool upper = pos[1] > ymax - P.eps;
    bool inlet = upper && pos[0] > P.inlet_x_lo && pos[0] < P.inlet_x_hi;
    if (inlet && dim == 3) inlet = pos[2] > P.inlet_z_lo && pos[2] < P.inlet_z_hi;
    if (inlet) rate[1] = Eval(P.inlet_rate);
}


// FvBaseLocalResidual::eval for element eid with derivatives with respect to local vertex `focus`
// (fvbaselocalresidual.hh:154-187): SCVF fluxes in edge order, the storage term of every vertex
// with its SCV volume, the boundary sub-faces, then division by each vertex's total control
// volume (UseVolumetricResidual).
static void vcfvEvalLocal(VCtx& C, const int64_t eid[3], const int64_t gv[8], const IQ* q[8], int focus, double dt,
                          int newtonIteration, Eval R[8][2], bool stashed = false) {
    const VGeom& g = C.geo;
    for (int v = 0; v < g.nv; ++v) { R[v][0] = Eval(0.0); R[v][1] = Eval(0.0); }
    for (int k = 0; k < g.ne; ++k) {
        Eval flux[2];
        vcfvFlux(C, q, k, focus, flux);
        double alpha = 1.0;  // extrusion factor
        alpha *= g.area[k];
        for (int a = 0; a < 2; ++a) flux[a] = flux[a] * alpha;
        for (int a = 0; a < 2; ++a) { R[g.ei[k]][a] += flux[a]; R[g.ej[k]][a] -= flux[a]; }
    }
    for (int v = 0; v < g.nv; ++v) {
        double scvVolume = g.scvVol * 1.0;
        Eval tmp[2];
        if (v == focus) storageOf<Eval>(*q[v], tmp);
        else { double t2[2]; storageOf<double>(*q[v], t2); tmp[0] = Eval(t2[0]); tmp[1] = Eval(t2[1]); }
        double tmp2[2];
        const int64_t G = gv[v];
        if (newtonIteration == 0 && !stashed) {
            if (!C.recycleStorage) {
                IQ qold = computeVIQ(C, G, C.sol[1].data());
                storageOf<double>(qold, tmp2);
            } else {
                tmp2[0] = tmp[0].v; tmp2[1] = tmp[1].v;
            }
            C.storageOld[2 * G] = tmp2[0]; C.storageOld[2 * G + 1] = tmp2[1];
        } else {
            tmp2[0] = C.storageOld[2 * G]; tmp2[1] = C.storageOld[2 * G + 1];
        }
        for (int a = 0; a < 2; ++a) {
            tmp[a] -= Eval(tmp2[a]);
            tmp[a] *= Eval(scvVolume / dt);
            R[v][a] += tmp[a];
        }
    }
    // boundary sub-faces (intersection order, then the face's vertices)
    for (int f = 0; f < g.nf; ++f) {
        const int a = g.faxis[f];
        const bool onB = g.fside[f] == 0 ? eid[a] == 0 : eid[a] == C.n[a] - 1;
        if (!onB) continue;
        for (int m = 0; m < g.nfv; ++m) {
            const int v = g.fv[f][m];
            Eval rate[2];
            vcfvBoundaryRate(C, eid, f, m, *q[v], v, gv[v], v == focus, rate);
            for (int e = 0; e < 2; ++e) { rate[e] = rate[e] * (g.barea[f][m] * 1.0); R[v][e] += rate[e]; }
        }
    }
    for (int v = 0; v < g.nv; ++v)
        for (int a = 0; a < 2; ++a) R[v][a] /= C.totVol[gv[v]];
}

static void vcfvBuildPattern(VCtx& C) {
    // createMatrix_: vertex rows couple to every vertex of the elements they belong to
    C.rowPtr.assign(C.NV + 1, 0);
    std::vector<int32_t> cols;
    for (int64_t v = 0; v < C.NV; ++v) {
        int64_t id[3]; C.vijk(v, id);
        for (int64_t dk = (C.dim == 3 ? -1 : 0); dk <= (C.dim == 3 ? 1 : 0); ++dk)
            for (int64_t dj = -1; dj <= 1; ++dj)
                for (int64_t di = -1; di <= 1; ++di) {
                    int64_t i = id[0] + di, j = id[1] + dj, k = id[2] + dk;
                    if (i < 0 || j < 0 || k < 0 || i >= C.nvx[0] || j >= C.nvx[1] || k >= C.nvx[2]) continue;
                    cols.push_back((int32_t)C.vindex(i, j, k));
                }
        C.rowPtr[v + 1] = (int32_t)cols.size();
    }
    C.colIdx = std::move(cols);
    C.blocks.assign(C.colIdx.size() * 4, 0.0);
}

static int32_t vcfvBlockPos(const VCtx& C, int64_t row, int64_t col) {
    for (int32_t q = C.rowPtr[row]; q < C.rowPtr[row + 1]; ++q) if (C.colIdx[q] == col) return q;
    return -1;
}

// FvBaseLinearizer::linearize_ with FvBaseAdLocalLinearizer (fvbaseadlocallinearizer.hh:178-204):
// per element, the intensive quantities of its vertices, then one evaluation of the local residual
// per focus vertex, and the scatter residual_[globI] += r_i, J[globJ][globI] += dR_j / dx_i of
// linearizeElement_ (fvbaselinearizer.hh:483-512), elements in index order.
static double vcfvLinearize(VCtx& C, double dt, int newtonIteration) {
    std::fill(C.resid.begin(), C.resid.end(), 0.0);
    std::fill(C.blocks.begin(), C.blocks.end(), 0.0);
    C.iqCache.resize(C.NV);
    const double* x = C.sol[0].data();
    parallelFor(C.nthreads, C.NV, [&](int64_t b, int64_t e, int) {
        for (int64_t v = b; v < e; ++v) C.iqCache[v] = computeVIQ(C, v, x);
    });
    const VGeom& g = C.geo;
    for (int64_t e = 0; e < C.NE; ++e) {
        int64_t eid[3]; C.eijk(e, eid);
        int64_t gv[8];
        const IQ* q[8];
        for (int v = 0; v < g.nv; ++v) { gv[v] = C.evert(eid, v); q[v] = &C.iqCache[gv[v]]; }
        double res[8][2];
        double jac[8][8][4];  // [dof][focus][eq*2+pv]
        if (C.fd) {
            // FvBaseFdLocalLinearizer (fvbasefdlocallinearizer.hh:221-237, 393-453): the local
            // residual at the primary variables, then, per focus vertex and primary variable, at the
            // deflected variable (only that vertex's intensive quantities re-evaluated, the storage
            // cache read, not written), eps = BaseEpsilon / primaryVarWeight
            Eval R0[8][2];
            vcfvEvalLocal(C, eid, gv, q, -1, dt, newtonIteration, R0);
            for (int f = 0; f < g.nv; ++f)
                for (int a = 0; a < 2; ++a) res[f][a] = R0[f][a].v;
            const double baseEps = std::max(0.9123e-10, std::numeric_limits<double>::epsilon() * 1.23e3);
            for (int f = 0; f < g.nv; ++f) {
                const IQ* qd[8];
                for (int w = 0; w < g.nv; ++w) qd[w] = q[w];
                for (int pv = 0; pv < 2; ++pv) {
                    const double pvWeight = pv == 0 ? 10 / C.refPressure : 1.0;
                    const double eps = baseEps / pvWeight;
                    double priVars[2] = {C.sol[0][2 * gv[f]], C.sol[0][2 * gv[f] + 1]};
                    double delta = 0.0;
                    double deriv[8][2];
                    Eval Rp[8][2];
                    if (C.fdMethod >= 0) {
                        priVars[pv] += eps;
                        delta += eps;
                        IQ qf = computeVIQAt(C, gv[f], priVars[0], priVars[1]);
                        qd[f] = &qf;
                        vcfvEvalLocal(C, eid, gv, qd, -1, dt, newtonIteration, Rp, true);
                        for (int d = 0; d < g.nv; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] = Rp[d][a].v;
                    } else {
                        for (int d = 0; d < g.nv; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] = R0[d][a].v;
                    }
                    if (C.fdMethod <= 0) {
                        priVars[pv] -= delta + eps;
                        delta += eps;
                        IQ qf = computeVIQAt(C, gv[f], priVars[0], priVars[1]);
                        qd[f] = &qf;
                        vcfvEvalLocal(C, eid, gv, qd, -1, dt, newtonIteration, Rp, true);
                        for (int d = 0; d < g.nv; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] -= Rp[d][a].v;
                    } else {
                        for (int d = 0; d < g.nv; ++d) for (int a = 0; a < 2; ++a) deriv[d][a] -= R0[d][a].v;
                    }
                    qd[f] = q[f];
                    for (int d = 0; d < g.nv; ++d)
                        for (int eq = 0; eq < 2; ++eq) jac[d][f][2 * eq + pv] = deriv[d][eq] / delta;
                }
            }
        } else
        for (int f = 0; f < g.nv; ++f) {
            Eval R[8][2];
            vcfvEvalLocal(C, eid, gv, q, f, dt, newtonIteration, R);
            for (int a = 0; a < 2; ++a) res[f][a] = R[f][a].v;
            for (int d = 0; d < g.nv; ++d)
                for (int eq = 0; eq < 2; ++eq)
                    for (int pv = 0; pv < 2; ++pv) jac[d][f][2 * eq + pv] = R[d][eq].d[pv];
        }
        for (int i = 0; i < g.nv; ++i) {
            const int64_t gi = gv[i];
            for (int a = 0; a < 2; ++a) C.resid[2 * gi + a] += res[i][a];
            for (int d = 0; d < g.nv; ++d) {
                int32_t pos = vcfvBlockPos(C, gv[d], gi);
                double* B = &C.blocks[4 * (size_t)pos];
                for (int t = 0; t < 4; ++t) B[t] += jac[d][i][t];
            }
        }
    }
    double err = 0.0;
    for (int64_t v = 0; v < C.NV; ++v) {
        double a = std::abs(C.resid[2 * v]), b = std::abs(C.resid[2 * v + 1]);
        if (!std::isfinite(a) || !std::isfinite(b)) return std::numeric_limits<double>::infinity();
        err = std::max(err, std::max(a, b));
    }
    return err;
}

static Bcrs vcfvMatrix(const VCtx& C) {
    Bcrs A; A.n = C.NV; A.rp = C.rowPtr; A.ci = C.colIdx; A.v = C.blocks; A.findDiag();
    return A;
}

}  // namespace orc

using namespace orc;

struct orc_ctx { Ctx C; };

extern "C" {

orc_ctx* orc_create(const ewg_grid* g, const ewg_problem* p, const double* perm, int nthreads) {
    orc_ctx* o = new orc_ctx();
    Ctx& C = o->C;
    C.dim = g->dim;
    C.n[0] = g->nx; C.n[1] = g->ny; C.n[2] = g->dim == 3 ? g->nz : 1;
    C.L[0] = g->lx; C.L[1] = g->ly; C.L[2] = g->dim == 3 ? g->lz : 1.0;
    for (int a = 0; a < 3; ++a) C.h[a] = C.L[a] / C.n[a];
    C.kOrigin = g->dim == 3 ? g->k_origin : 0;
    C.N = (int64_t)C.n[0] * C.n[1] * C.n[2];
    C.prob = *p;
    C.law[0] = makeLaw(p->outer);
    C.law[1] = makeLaw(p->lens);
    C.perm.assign(perm, perm + C.N);
    C.inLens.resize(C.N);
    for (int64_t c = 0; c < C.N; ++c) { double x[3]; C.center(c, x); C.inLens[c] = C.isInLens(x) ? 1 : 0; }
    C.sol[0].assign(2 * C.N, 0.0); C.sol[1].assign(2 * C.N, 0.0);
    C.storageOld.assign(2 * C.N, 0.0);
    C.resid.assign(2 * C.N, 0.0);
    C.nthreads = std::max(1, nthreads);
    buildPattern(C);
    return o;
}
void orc_destroy(orc_ctx* c) { delete c; }
const char* orc_last_error(const orc_ctx* c) { return c->C.err.c_str(); }
int64_t orc_num_cells(const orc_ctx* c) { return c->C.N; }
int64_t orc_num_blocks(const orc_ctx* c) { return (int64_t)c->C.colIdx.size(); }
void orc_set_recycle_first_iteration_storage(orc_ctx* c, int on) { c->C.recycleStorage = on != 0; }
// kind 0: AD, 1: finite differences with NumericDifferenceMethod `method`
void orc_set_local_linearizer(orc_ctx* c, int kind, int method) { c->C.fd = kind == 1; c->C.fdMethod = method; }

void orc_set_solution(orc_ctx* c, int t, const double* x) { c->C.sol[t].assign(x, x + 2 * c->C.N); }
void orc_get_solution(const orc_ctx* c, int t, double* x) { std::memcpy(x, c->C.sol[t].data(), sizeof(double) * 2 * c->C.N); }

// LensProblem::initial (lensproblem.hh:545-578) + assignNaive
void orc_apply_initial_solution(orc_ctx* o) {
    Ctx& C = o->C;
    double ymax = C.L[1];
    for (int64_t c = 0; c < C.N; ++c) {
        double x[3]; C.center(c, x);
        double depth = ymax - x[1];
        double densityW = C.prob.rho_w;
        double pw = C.prob.p_ref - densityW * C.gravity(1) * depth;
        C.sol[0][2 * c] = pw; C.sol[0][2 * c + 1] = 1.0;
    }
    C.sol[1] = C.sol[0];
}
void orc_advance_time_level(orc_ctx* o) { o->C.sol[1] = o->C.sol[0]; }

void orc_update_begin(orc_ctx* o) { o->C.refPressure = o->C.sol[0][0]; }
// updateBegin with the caller's reference pressure (a z-slab takes the whole grid's)
// updateBegin with a caller-given reference pressure; like ewg_set_reference_pressure it rejects a
// value that is not positive and finite (returns 1 and leaves the stored pressure unchanged)
int orc_set_reference_pressure(orc_ctx* o, double p) {
    if (!(p > 0) || !std::isfinite(p)) {
        o->C.err = "set_reference_pressure: p_ref must be positive and finite";
        return 1;
    }
    o->C.refPressure = p;
    return 0;
}
int orc_linearize(orc_ctx* o, double dt, int it, double* error) {
    // a context that never ran updateBegin takes the reference pressure of the current iterate
    if (o->C.fd && !(o->C.refPressure > 0)) o->C.refPressure = o->C.sol[0][0];
    try {
        double e = linearize(o->C, dt, it);
        if (error) *error = e;
        return 0;
    } catch (const std::exception& ex) { o->C.err = ex.what(); return 1; }
}
void orc_get_residual(const orc_ctx* o, double* r) { std::memcpy(r, o->C.resid.data(), sizeof(double) * 2 * o->C.N); }
void orc_get_jacobian_bcrs(const orc_ctx* o, int32_t* rp, int32_t* ci, double* b) {
    const Ctx& C = o->C;
    if (rp) std::memcpy(rp, C.rowPtr.data(), sizeof(int32_t) * C.rowPtr.size());
    if (ci) std::memcpy(ci, C.colIdx.data(), sizeof(int32_t) * C.colIdx.size());
    if (b) std::memcpy(b, C.blocks.data(), sizeof(double) * C.blocks.size());
}
void orc_set_jacobian_blocks(orc_ctx* o, const double* b) { o->C.blocks.assign(b, b + o->C.blocks.size()); }
void orc_set_residual(orc_ctx* o, const double* r) { o->C.resid.assign(r, r + 2 * o->C.N); }

int orc_fd_jacobian(orc_ctx* o, double dt, double* out) {
    Ctx& C = o->C;
    try {
        std::vector<double> x0 = C.sol[0];
        std::vector<double> so = C.storageOld;
        linearize(C, dt, 1);  // storage cache already filled by the caller
        std::vector<double> r0 = C.resid;
        std::vector<double> blocks(C.blocks.size(), 0.0);
        for (int64_t col = 0; col < C.N; ++col) {
            for (int pv = 0; pv < 2; ++pv) {
                double base = x0[2 * col + pv];
                double eps = pv == 0 ? 1e-2 : 1e-8;  // pressure ~1e5 Pa, saturation ~1
                std::vector<double>& x = C.sol[0];
                x[2 * col + pv] = base + eps;
                linearize(C, dt, 1);
                std::vector<double> rp = C.resid;
                x[2 * col + pv] = base - eps;
                linearize(C, dt, 1);
                std::vector<double> rm = C.resid;
                x[2 * col + pv] = base;
                // rows that see this column: the column's own row and its neighbours' rows
                for (int64_t row = 0; row < C.N; ++row) {
                    for (int32_t q = C.rowPtr[row]; q < C.rowPtr[row + 1]; ++q) {
                        if (C.colIdx[q] != col) continue;
                        for (int eq = 0; eq < 2; ++eq)
                            blocks[4 * (size_t)q + 2 * eq + pv] = (rp[2 * row + eq] - rm[2 * row + eq]) / (2 * eps);
                    }
                }
            }
        }
        C.sol[0] = x0;
        C.storageOld = so;
        linearize(C, dt, 1);
        std::memcpy(out, blocks.data(), sizeof(double) * blocks.size());
        return 0;
    } catch (const std::exception& ex) { C.err = ex.what(); return 1; }
}

int orc_solve(orc_ctx* o, const ewg_solve_opts* so, int ordering, double* dx, int* iterations, double* finalRes) {
    Ctx& C = o->C;
    try {
        Bcrs A = systemMatrix(C);
        Precond M; M.kind = so->precond; M.ordering = ordering; M.w = so->preconditioner_relaxation;
        M.setup(C, A);
        Criterion crit{so->linear_solver_tolerance, so->linear_solver_abs_tolerance, so->linear_solver_max_error};
        std::vector<double> x;
        int it = 0, restarts = 0;
        bool ok = bicgstab(A, M, C.resid, x, crit, so->linear_solver_max_iterations,
                           so->restart_on_breakdown != 0, so->verify_true_residual != 0, &it, &restarts);
        if (dx) std::memcpy(dx, x.data(), sizeof(double) * x.size());
        if (iterations) *iterations = it;
        if (finalRes) *finalRes = crit.resErr;
        return ok ? 0 : EWG_ERR_NOT_CONVERGED;
    } catch (const BreakdownError& ex) { C.err = ex.what(); return EWG_ERR_BREAKDOWN; }
    catch (const std::exception& ex) { C.err = ex.what(); return EWG_ERR_INVALID; }
}

int orc_apply_preconditioner(orc_ctx* o, const ewg_solve_opts* so, int ordering, const double* b, double* y) {
    Ctx& C = o->C;
    try {
        Bcrs A = systemMatrix(C);
        Precond M; M.kind = so->precond; M.ordering = ordering; M.w = so->preconditioner_relaxation;
        M.setup(C, A);
        M.apply(b, y);
        return 0;
    } catch (const std::exception& ex) { C.err = ex.what(); return 1; }
}

void orc_apply_jacobian(const orc_ctx* o, const double* x, double* y) {
    Bcrs A = systemMatrix(o->C);
    A.mv(x, y);
}

// NewtonMethod::apply at a fixed time-step size
int orc_newton_apply(orc_ctx* o, double dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                     int ordering, int* newtonIts, int* linIts, double* errorOut) {
    Ctx& C = o->C;
    int numIterations = 0, linTotal = 0;
    double error = 1e100, lastError = 1e100;
    auto converged = [&]() { return error <= no->newton_tolerance; };
    auto proceed = [&]() {
        if (numIterations < 1) return true;
        if (converged()) return false;
        if (numIterations >= no->newton_max_iterations) return error * 4.0 < lastError;
        return true;
    };
    int status = 0;
    // ImmiscibleModel::updateBegin, called before every Newton solve: p_w of the first DOF
    C.refPressure = C.sol[0][0];
    try {
        while (proceed()) {
            lastError = error;
            double e = linearize(C, dt, numIterations);
            // preSolve_: max-norm of the residual, eqWeight == 1
            lastError = error;
            error = e;
            if (error > no->newton_max_error) throw std::runtime_error("Newton: error above NewtonMaxError");
            if (!proceed()) { ++numIterations; break; }
            std::vector<double> dx(2 * C.N);
            int it = 0;
            double fr = 0;
            int rc = orc_solve(o, so, ordering, dx.data(), &it, &fr);
            linTotal += it;
            if (rc != 0) { status = rc; break; }
            double one = 0.0;
            for (double v : dx) one += std::abs(v);
            if (!std::isfinite(one)) throw std::runtime_error("Non-finite update!");
            for (int64_t i = 0; i < 2 * C.N; ++i) C.sol[0][i] -= dx[i];
            ++numIterations;
        }
    } catch (const std::exception& ex) { C.err = ex.what(); status = EWG_ERR_NONFINITE; }
    if (newtonIts) *newtonIts = numIterations;
    if (linIts) *linIts = linTotal;
    if (errorOut) *errorOut = error;
    if (status) return status;
    return converged() ? 0 : EWG_ERR_NOT_CONVERGED;
}

double orc_residual_norm(orc_ctx* o, const double* x, double dt) {
    Ctx& C = o->C;
    std::vector<double> keep = C.sol[0];
    std::vector<double> r = C.resid; std::vector<double> b = C.blocks;
    C.sol[0].assign(x, x + 2 * C.N);
    double e = 0.0;
    try { e = linearize(C, dt, 1); } catch (...) { e = std::numeric_limits<double>::infinity(); }
    C.sol[0] = keep; C.resid = r; C.blocks = b;
    return e;
}

void orc_material_eval(const ewg_material* m, double sw, double* out) {
    Law L = makeLaw(*m);
    Eval S = Eval::variable(sw, 1);
    Eval pc[2], kr[2];
    capillaryPressures(pc, L, S);
    relativePermeabilities(kr, L, S);
    out[0] = pc[1].v; out[1] = pc[1].d[1];
    out[2] = kr[0].v; out[3] = kr[0].d[1];
    out[4] = kr[1].v; out[5] = kr[1].d[1];
}

void orc_global_storage(const orc_ctx* o, int t, double* out) {
    const Ctx& C = o->C;
    out[0] = out[1] = 0.0;
    for (int64_t c = 0; c < C.N; ++c) {
        IQ q = computeIQ(C, c, C.sol[t].data(), false);
        double s[2]; storageOf<double>(q, s);
        out[0] += s[0] * C.vol(); out[1] += s[1] * C.vol();
    }
}

void orc_boundary_rates(orc_ctx* o, double* out) {
    Ctx& C = o->C;
    out[0] = out[1] = 0.0;
    Face f[6];
    for (int64_t c = 0; c < C.N; ++c) {
        C.faces(c, f);
        IQ q = computeIQ(C, c, C.sol[0].data(), true);
        for (int k = 0; k < C.numFaces(); ++k) {
            if (f[k].nbr >= 0) continue;
            Eval rate[2]; int kind;
            boundaryRate(C, c, f[k], q, rate, &kind);
            out[0] += rate[0].v * C.area(f[k].axis);
            out[1] += rate[1].v * C.area(f[k].axis);
        }
    }
}

}  // extern "C"

// ---- vertex-centred discretization -------------------------------------------------------------

struct orc_vcfv { VCtx C; };

extern "C" {

// perm: one permeability per vertex, vertices numbered x fastest ((nx+1) x (ny+1) [x (nz+1)])
orc_vcfv* orc_vcfv_create(const ewg_grid* g, const ewg_problem* p, const double* perm, int nthreads) {
    orc_vcfv* o = new orc_vcfv();
    VCtx& C = o->C;
    C.dim = g->dim;
    C.n[0] = g->nx; C.n[1] = g->ny; C.n[2] = g->dim == 3 ? g->nz : 1;
    C.L[0] = g->lx; C.L[1] = g->ly; C.L[2] = g->dim == 3 ? g->lz : 1.0;
    for (int a = 0; a < 3; ++a) C.h[a] = C.L[a] / C.n[a];
    for (int a = 0; a < 3; ++a) C.nvx[a] = a < C.dim ? C.n[a] + 1 : 1;
    C.NE = (int64_t)C.n[0] * C.n[1] * C.n[2];
    C.NV = (int64_t)C.nvx[0] * C.nvx[1] * C.nvx[2];
    C.prob = *p;
    C.law[0] = makeLaw(p->outer);
    C.law[1] = makeLaw(p->lens);
    C.geo = makeVGeom(C.dim, C.h);
    C.perm.assign(perm, perm + C.NV);
    C.inLens.resize(C.NV);
    for (int64_t v = 0; v < C.NV; ++v) { double x[3]; C.vpos(v, x); C.inLens[v] = C.isInLens(x) ? 1 : 0; }
    // dofTotalVolume: the SCV volumes summed over the elements in index order
    C.totVol.assign(C.NV, 0.0);
    for (int64_t e = 0; e < C.NE; ++e) {
        int64_t eid[3]; C.eijk(e, eid);
        for (int v = 0; v < C.geo.nv; ++v) C.totVol[C.evert(eid, v)] += C.geo.scvVol * 1.0;
    }
    C.sol[0].assign(2 * C.NV, 0.0); C.sol[1].assign(2 * C.NV, 0.0);
    C.storageOld.assign(2 * C.NV, 0.0);
    C.resid.assign(2 * C.NV, 0.0);
    C.nthreads = std::max(1, nthreads);
    vcfvBuildPattern(C);
    return o;
}
void orc_vcfv_destroy(orc_vcfv* o) { delete o; }
const char* orc_vcfv_last_error(const orc_vcfv* o) { return o->C.err.c_str(); }
int64_t orc_vcfv_num_dofs(const orc_vcfv* o) { return o->C.NV; }
int64_t orc_vcfv_num_blocks(const orc_vcfv* o) { return (int64_t)o->C.colIdx.size(); }
void orc_vcfv_set_solution(orc_vcfv* o, int t, const double* x) { o->C.sol[t].assign(x, x + 2 * o->C.NV); }
void orc_vcfv_get_solution(const orc_vcfv* o, int t, double* x) {
    std::memcpy(x, o->C.sol[t].data(), sizeof(double) * 2 * o->C.NV);
}
// LensProblem::initial at the vertex positions
void orc_vcfv_apply_initial_solution(orc_vcfv* o) {
    VCtx& C = o->C;
    for (int64_t v = 0; v < C.NV; ++v) {
        double x[3]; C.vpos(v, x);
        double depth = C.L[1] - x[1];
        C.sol[0][2 * v] = C.prob.p_ref - C.prob.rho_w * C.gravity(1) * depth;
        C.sol[0][2 * v + 1] = 1.0;
    }
    C.sol[1] = C.sol[0];
}
void orc_vcfv_advance_time_level(orc_vcfv* o) { o->C.sol[1] = o->C.sol[0]; }
// kind 0: AD, 1: finite differences with NumericDifferenceMethod `method`
void orc_vcfv_set_local_linearizer(orc_vcfv* o, int kind, int method) { o->C.fd = kind == 1; o->C.fdMethod = method; }
// ImmiscibleModel::updateBegin: the reference pressure of the FD pressure weight
void orc_vcfv_update_begin(orc_vcfv* o) { o->C.refPressure = o->C.sol[0][0]; }
void orc_vcfv_total_volumes(const orc_vcfv* o, double* out) {
    std::memcpy(out, o->C.totVol.data(), sizeof(double) * o->C.NV);
}
int orc_vcfv_linearize(orc_vcfv* o, double dt, int it, double* error) {
    if (o->C.fd && !(o->C.refPressure > 0)) o->C.refPressure = o->C.sol[0][0];
    try {
        double e = vcfvLinearize(o->C, dt, it);
        if (error) *error = e;
        return 0;
    } catch (const std::exception& ex) { o->C.err = ex.what(); return 1; }
}
void orc_vcfv_get_residual(const orc_vcfv* o, double* r) {
    std::memcpy(r, o->C.resid.data(), sizeof(double) * 2 * o->C.NV);
}
void orc_vcfv_get_jacobian_bcrs(const orc_vcfv* o, int32_t* rp, int32_t* ci, double* b) {
    const VCtx& C = o->C;
    if (rp) std::memcpy(rp, C.rowPtr.data(), sizeof(int32_t) * C.rowPtr.size());
    if (ci) std::memcpy(ci, C.colIdx.data(), sizeof(int32_t) * C.colIdx.size());
    if (b) std::memcpy(b, C.blocks.data(), sizeof(double) * C.blocks.size());
}

// NewtonMethod::apply at a fixed time-step size with BiCGStab and the block ILU(0) (natural order,
// or the parity-colour order of the device) or block Jacobi preconditioner of so->precond
int orc_vcfv_newton_apply(orc_vcfv* o, double dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                          int ordering, int* newtonIts, int* linIts, double* errorOut) {
    VCtx& C = o->C;
    static const Ctx kNoGrid{};
    int numIterations = 0, linTotal = 0;
    double error = 1e100, lastError = 1e100;
    auto converged = [&]() { return error <= no->newton_tolerance; };
    auto proceed = [&]() {
        if (numIterations < 1) return true;
        if (converged()) return false;
        if (numIterations >= no->newton_max_iterations) return error * 4.0 < lastError;
        return true;
    };
    int status = 0;
    C.refPressure = C.sol[0][0];  // ImmiscibleModel::updateBegin before every Newton solve
    try {
        while (proceed()) {
            double e = vcfvLinearize(C, dt, numIterations);
            lastError = error;
            error = e;
            if (error > no->newton_max_error) throw std::runtime_error("Newton: error above NewtonMaxError");
            if (!proceed()) { ++numIterations; break; }
            Bcrs A = vcfvMatrix(C);
            Precond M; M.kind = so->precond; M.ordering = ordering; M.w = so->preconditioner_relaxation;
            if (ordering == ORC_ORDER_COLOURS) {
                M.colourOf.resize(C.NV);
                for (int64_t v = 0; v < C.NV; ++v) {
                    int64_t id[3]; C.vijk(v, id);
                    M.colourOf[v] = (int8_t)((id[0] & 1) + 2 * (id[1] & 1) + 4 * (id[2] & 1));
                }
            }
            M.setup(kNoGrid, A);
            Criterion crit{so->linear_solver_tolerance, so->linear_solver_abs_tolerance, so->linear_solver_max_error};
            std::vector<double> dx;
            int it = 0, restarts = 0;
            bool ok = bicgstab(A, M, C.resid, dx, crit, so->linear_solver_max_iterations,
                               so->restart_on_breakdown != 0, so->verify_true_residual != 0, &it, &restarts);
            linTotal += it;
            if (!ok) { status = EWG_ERR_NOT_CONVERGED; break; }
            double one = 0.0;
            for (double v : dx) one += std::abs(v);
            if (!std::isfinite(one)) throw std::runtime_error("Non-finite update!");
            for (int64_t i = 0; i < 2 * C.NV; ++i) C.sol[0][i] -= dx[i];
            ++numIterations;
        }
    } catch (const BreakdownError& ex) { C.err = ex.what(); status = EWG_ERR_BREAKDOWN; }
    catch (const std::exception& ex) { C.err = ex.what(); status = EWG_ERR_NONFINITE; }
    if (newtonIts) *newtonIts = numIterations;
    if (linIts) *linIts = linTotal;
    if (errorOut) *errorOut = error;
    if (status) return status;
    return converged() ? 0 : EWG_ERR_NOT_CONVERGED;
}

// total mass of each phase (storage x total control volume) at time level t
void orc_vcfv_global_storage(const orc_vcfv* o, int t, double* out) {
    const VCtx& C = o->C;
    out[0] = out[1] = 0.0;
    for (int64_t v = 0; v < C.NV; ++v) {
        IQ q = computeVIQ(C, v, C.sol[t].data());
        double s[2]; storageOf<double>(q, s);
        out[0] += s[0] * C.totVol[v]; out[1] += s[1] * C.totVol[v];
    }
}

// sum of boundary mass rates x area over all boundary sub-faces at the current solution
void orc_vcfv_boundary_rates(orc_vcfv* o, double* out) {
    VCtx& C = o->C;
    out[0] = out[1] = 0.0;
    const VGeom& g = C.geo;
    for (int64_t e = 0; e < C.NE; ++e) {
        int64_t eid[3]; C.eijk(e, eid);
        for (int f = 0; f < g.nf; ++f) {
            const int a = g.faxis[f];
            const bool onB = g.fside[f] == 0 ? eid[a] == 0 : eid[a] == C.n[a] - 1;
            if (!onB) continue;
            for (int m = 0; m < g.nfv; ++m) {
                const int v = g.fv[f][m];
                int64_t gv = C.evert(eid, v);
                IQ q = computeVIQ(C, gv, C.sol[0].data());
                Eval rate[2];
                vcfvBoundaryRate(C, eid, f, m, q, v, gv, false, rate);
                out[0] += rate[0].v * g.barea[f][m];
                out[1] += rate[1].v * g.barea[f][m];
            }
        }
    }
}

// the local geometry of the structured element: for each SCVF k (i, j, ip[3], nrm[3], area) and the
// P1 gradients G[k][v][3]; scv volume
void orc_vcfv_geometry(const orc_vcfv* o, int32_t* ij, double* ip, double* nrm, double* area, double* G,
                       double* scvVol) {
    const VGeom& g = o->C.geo;
    for (int k = 0; k < g.ne; ++k) {
        ij[2 * k] = g.ei[k]; ij[2 * k + 1] = g.ej[k];
        for (int d = 0; d < 3; ++d) { ip[3 * k + d] = g.ip[k][d]; nrm[3 * k + d] = g.nrm[k][d]; }
        area[k] = g.area[k];
        for (int v = 0; v < g.nv; ++v)
            for (int d = 0; d < 3; ++d) G[(k * 8 + v) * 3 + d] = g.G[k][v][d];
    }
    *scvVol = g.scvVol;
}

}  // extern "C"
