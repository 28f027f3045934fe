// Device pieces of the BiCGStab / block-ILU(0) solver shared by the single-problem solver
// (ewg_solver.cu) and the batched ensemble (ewg_ensemble.cu): the solver state of
// BiCGStabSolver::apply / CombinedCriterion (linear/bicgstabsolver.hh:116-326,
// linear/combinedcriterion.hh:112-205), 2x2 block helpers, and the per-row arithmetic of the
// band-stored SpMV and of the red-black block ILU(0) (dune-istl bilu0_decomposition /
// bilu_backsolve restricted to the two-colour ordering).
#pragma once

#include <math_constants.h>

#include <cfloat>

#include "ewg_internal.cuh"

namespace ewg {

constexpr int kSolBlock = 256;

// Programmatic dependent launch. A kernel launched with EWG_LAUNCH_PDL may be scheduled while the
// kernel before it in the stream is still finishing; its first statement, pdl_enter, waits until
// that kernel has completed with its writes visible and then lets the next kernel be scheduled.
// So a PDL kernel completes only after its predecessor did, and nothing it reads or writes can
// race with an earlier kernel; what overlaps is the launch and block setup with the tail of the
// previous kernel. In a kernel launched without the attribute both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
constexpr int kMaxRed = 4;

enum BiStatus { ST_RUNNING = 0, ST_CONVERGED = 1, ST_FAILED = 2, ST_BREAKDOWN = 3, ST_MAXITER = 4 };

struct BiState {
    double rho, alpha, omega, rho_i, beta;
    double r0r0;
    double resErr, lastResErr, initResErr;
    double relTol, absTol, maxRes;
    double w;           // preconditioner relaxation
    int status;
    int iter;
    int restarts;
    int maxIter;
    int restartOnBreakdown;
    int restartPending;
    int stagnates;
    int replacements;
    int verifyTrue;
};

template <typename T> struct V2T;
template <> struct V2T<double> { using type = double2; };
template <> struct V2T<float> { using type = float2; };

// NaN-propagating |x| for max reductions: NaN compares false, so map it to +inf
__device__ __forceinline__ double absn(double x) { return x == x ? fabs(x) : CUDART_INF; }

// ---- 2x2 helpers --------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ void load_block(const T* __restrict__ A, int64_t stride, int band, int64_t s, double b[4]) {
    const T* p = A + (int64_t)band * 4 * stride + s;
    b[0] = (double)p[0];
    b[1] = (double)p[stride];
    b[2] = (double)p[2 * stride];
    b[3] = (double)p[3 * stride];
}
template <typename T>
__device__ __forceinline__ void store4(T* __restrict__ A, int64_t stride, int plane4, int64_t s, const double b[4]) {
    T* p = A + (int64_t)plane4 * 4 * stride + s;
    p[0] = (T)b[0];
    p[stride] = (T)b[1];
    p[2 * stride] = (T)b[2];
    p[3 * stride] = (T)b[3];
}
__device__ __forceinline__ bool inv2(const double a[4], double o[4]) {
    double det = a[0] * a[3] - a[1] * a[2];
    if (det == 0.0 || !isfinite(det)) return false;
    double di = 1.0 / det;
    o[0] = a[3] * di;
    o[1] = -a[1] * di;
    o[2] = -a[2] * di;
    o[3] = a[0] * di;
    return true;
}
__device__ __forceinline__ void mul2(const double a[4], const double b[4], double o[4]) {
    double t0 = a[0] * b[0] + a[1] * b[2], t1 = a[0] * b[1] + a[1] * b[3];
    double t2 = a[2] * b[0] + a[3] * b[2], t3 = a[2] * b[1] + a[3] * b[3];
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}

// bands in ascending column order of a natural-order BCRS row, without the diagonal
__host__ __device__ inline int lower_upper_band(int dim, int q) {
    // 3D: -z -y -x +x +y +z ; 2D: -y -x +x +y
    return dim == 3 ? (q == 0 ? 5 : q == 1 ? 3 : q == 2 ? 1 : q == 3 ? 2 : q == 4 ? 4 : 6)
                    : (q == 0 ? 3 : q == 1 ? 1 : q == 2 ? 2 : 4);
}

__device__ __forceinline__ int64_t nbr_of_band(const Phys& P, int col, int64_t h, const CellIdx& ci, int band) {
    return neighbour_split(P, col, h, ci, (band - 1) >> 1, (band - 1) & 1);
}

// ---- preconditioner rows ---------------------------------------------------------------------

// Dinv(s) = inv(A_ss); false if the block is singular (Dinv(s) = 0 then)
template <typename TM>
__device__ __forceinline__ bool diag_inverse_row(int64_t N, const TM* __restrict__ A, TM* __restrict__ Dinv, int64_t s) {
    double a[4], o[4];
    load_block(A, N, 0, s, a);
    const bool ok = inv2(a, o);
    if (!ok) o[0] = o[1] = o[2] = o[3] = 0.0;
    store4(Dinv, N, 0, s, o);
    return ok;
}

// black row h: L_bk = A_bk inv(D_k) in ascending column order, D_b' = A_bb - sum L_bk A_kb
template <typename TM>
__device__ __forceinline__ bool ilu_black_factor_row(const Phys& P, const TM* __restrict__ A, TM* __restrict__ Dinv,
                                                     TM* __restrict__ L, int64_t h) {
    const int nOff = 2 * P.dim;
    const int64_t s = P.Nh + h;
    const CellIdx ci = cell_of(P, 1, h);
    double D[4];
    load_block(A, P.N, 0, s, D);
    for (int q = 0; q < nOff; ++q) {
        const int band = lower_upper_band(P.dim, q);
        const int64_t sk = nbr_of_band(P, 1, h, ci, band);
        double Lb[4] = {0.0, 0.0, 0.0, 0.0};
        if (sk >= 0) {
            double Abk[4], Dk[4], Akb[4], B[4];
            load_block(A, P.N, band, s, Abk);
            load_block(Dinv, P.N, 0, sk, Dk);
            mul2(Abk, Dk, Lb);
            load_block(A, P.N, opposite_band(band), sk, Akb);
            mul2(Lb, Akb, B);
            for (int t = 0; t < 4; ++t) D[t] -= B[t];
        }
        store4(L, P.Nh, band - 1, h, Lb);
    }
    double o[4];
    const bool ok = inv2(D, o);
    if (!ok) o[0] = o[1] = o[2] = o[3] = 0.0;
    store4(Dinv, P.N, 0, s, o);
    return ok;
}

// black row h of the forward sweep: y_b = w inv(D_b') (d_b - sum_k L_bk d_k)
template <typename TM, typename TV>
__device__ __forceinline__ void ilu_black_apply_row(const Phys& P, const TM* __restrict__ Dinv, const TM* __restrict__ L,
                                                    const typename V2T<TV>::type* __restrict__ d,
                                                    typename V2T<TV>::type* __restrict__ y, double w, int64_t h) {
    const int nOff = 2 * P.dim;
    const int64_t s = P.Nh + h;
    const CellIdx ci = cell_of(P, 1, h);
    auto ds = d[s];
    double r0 = (double)ds.x, r1 = (double)ds.y;
    for (int q = 0; q < nOff; ++q) {
        const int band = lower_upper_band(P.dim, q);
        const int64_t sk = nbr_of_band(P, 1, h, ci, band);
        if (sk < 0) continue;
        double Lb[4];
        load_block(L, P.Nh, band - 1, h, Lb);
        auto dk = d[sk];
        const double x0 = (double)dk.x, x1 = (double)dk.y;
        r0 -= Lb[0] * x0; r0 -= Lb[1] * x1;
        r1 -= Lb[2] * x0; r1 -= Lb[3] * x1;
    }
    double Di[4];
    load_block(Dinv, P.N, 0, s, Di);
    typename V2T<TV>::type out;
    out.x = (TV)(w * (Di[0] * r0 + Di[1] * r1));
    out.y = (TV)(w * (Di[2] * r0 + Di[3] * r1));
    y[s] = out;
}

// red row h after the black phase: y_r = w inv(D_r) (d_r - sum_b A_rb y_b / w), columns
// descending. With relaxation w != 1 the black values were scaled by w; the backward sweep of
// the reference runs on unscaled values and scales at the end, so the coupling term undoes it.
template <typename TM, typename TV>
__device__ __forceinline__ void ilu_red_apply_row(const Phys& P, const TM* __restrict__ A, const TM* __restrict__ Dinv,
                                                  const typename V2T<TV>::type* __restrict__ d,
                                                  typename V2T<TV>::type* __restrict__ y, double w, double winv,
                                                  int64_t h) {
    const int nOff = 2 * P.dim;
    const int64_t s = h;
    const CellIdx ci = cell_of(P, 0, h);
    auto ds = d[s];
    double r0 = (double)ds.x, r1 = (double)ds.y;
    for (int q = nOff - 1; q >= 0; --q) {
        const int band = lower_upper_band(P.dim, q);
        const int64_t sk = nbr_of_band(P, 0, h, ci, band);
        if (sk < 0) continue;
        double Ab[4];
        load_block(A, P.N, band, s, Ab);
        auto yk = y[sk];
        double x0 = (double)yk.x, x1 = (double)yk.y;
        if (w != 1.0) { x0 *= winv; x1 *= winv; }
        r0 -= Ab[0] * x0; r0 -= Ab[1] * x1;
        r1 -= Ab[2] * x0; r1 -= Ab[3] * x1;
    }
    double Di[4];
    load_block(Dinv, P.N, 0, s, Di);
    typename V2T<TV>::type out;
    out.x = (TV)(w * (Di[0] * r0 + Di[1] * r1));
    out.y = (TV)(w * (Di[2] * r0 + Di[3] * r1));
    y[s] = out;
}

// ---- SpMV row ----------------------------------------------------------------------------------

template <typename TM, typename TV>
__device__ __forceinline__ void spmv_row(const Phys& P, const TM* __restrict__ A,
                                         const typename V2T<TV>::type* __restrict__ x, int64_t s,
                                         double& a0, double& a1) {
    const int col = s >= P.Nh ? 1 : 0;
    const int64_t h = s - col * P.Nh;
    const CellIdx ci = cell_of(P, col, h);
    const int nOff = 2 * P.dim;
    a0 = 0.0; a1 = 0.0;
    const bool interior = ci.i > 0 && ci.i < P.nx - 1 && ci.j > 0 && ci.j < P.ny - 1 &&
                          (P.dim == 2 || (ci.k > 0 && ci.k < P.nz - 1));
    if (P.dim == 3 && interior) {
        // all seven blocks exist: issue every load before the arithmetic
        const int64_t base = (int64_t)(col ^ 1) * P.Nh;
        const int64_t nb[7] = {base + h - P.planeh, base + h - P.nxh, base + h - 1 + ci.b, s,
                               base + h + ci.b, base + h + P.nxh, base + h + P.planeh};
        const int bands[7] = {5, 3, 1, 0, 2, 4, 6};
        double B[7][4];
        double xv[7][2];
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            load_block(A, P.N, bands[q], s, B[q]);
            auto xk = x[nb[q]];
            xv[q][0] = (double)xk.x;
            xv[q][1] = (double)xk.y;
        }
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            a0 += B[q][0] * xv[q][0]; a0 += B[q][1] * xv[q][1];
            a1 += B[q][2] * xv[q][0]; a1 += B[q][3] * xv[q][1];
        }
        return;
    }
    // ascending columns: lower bands, diagonal, upper bands
    for (int q = 0; q <= nOff; ++q) {
        int band;
        int64_t sk;
        if (q == P.dim) { band = 0; sk = s; }
        else {
            band = lower_upper_band(P.dim, q < P.dim ? q : q - 1);
            sk = nbr_of_band(P, col, h, ci, band);
            if (sk < 0) continue;
        }
        double B[4];
        load_block(A, P.N, band, s, B);
        auto xk = x[sk];
        const double x0 = (double)xk.x, x1 = (double)xk.y;
        a0 += B[0] * x0; a0 += B[1] * x1;
        a1 += B[2] * x0; a1 += B[3] * x1;
    }
}

// ---- BiCGStab scalar updates (executed by one thread after a reduction) -------------------------

__device__ __forceinline__ void criterion_check(BiState* st) {
    // CombinedCriterion::converged / failed
    double red = st->resErr / fmax(1e-20, st->initResErr);
    bool conv = red <= st->relTol || st->resErr <= st->absTol;
    if (conv) { st->status = ST_CONVERGED; return; }
    if (st->stagnates || st->resErr > st->maxRes) st->status = ST_FAILED;
}

// top of a BiCGStab iteration: shadow restart, breakdown test, beta, rho
__device__ __forceinline__ void iteration_top(BiState* st, double rho_i, double rr) {
    const double breakdownEps = DBL_MIN * 1e10;
    if (st->iter >= st->maxIter) { st->status = ST_MAXITER; return; }
    if (st->restartOnBreakdown && fabs(rho_i) <= 1e-12 * sqrt(st->r0r0) * sqrt(rr)) {
        st->restartPending = 1;
        st->r0r0 = rr;
        rho_i = rr;
        st->rho = 1.0; st->alpha = 1.0; st->omega = 1.0;
        st->restarts += 1;
    }
    if (fabs(st->rho) <= breakdownEps || fabs(st->omega) <= breakdownEps) { st->status = ST_BREAKDOWN; return; }
    st->beta = (rho_i / st->rho) * (st->alpha / st->omega);
    st->rho = rho_i;
    st->rho_i = rho_i;
}

}  // namespace ewg
