// Preconditioned BiCGStab on the band-stored block Jacobian (linear/bicgstabsolver.hh:116-326,
// linear/combinedcriterion.hh:112-205, linear/parallelbasebackend.hh:301-338).
//
// Device design
//   * All vectors are 2-blocks per cell in red-black split order (see ewg_internal.cuh).
//   * Every BiCGStab scalar (rho, alpha, omega, the criterion errors, the status) lives in a
//     device-side state word. Each kernel ends with a deterministic grid reduction (fixed grid,
//     per-block partials, the last block to finish sums the partials in block order) and that
//     last block updates the scalars, so the host never sits between two kernels of an iteration.
//     The host reads the status only every few iterations; kernels launched after convergence
//     return immediately.
//   * Block ILU(0) in red-black order (colour 0 first). Red rows have only black neighbours, so
//     the factorisation only changes black rows: L_bk = A_bk inv(D_k), D_b' = A_bb - sum L_bk A_kb
//     (dune-istl bilu0_decomposition restricted to this ordering). Each sweep of
//     bilu_backsolve becomes one fully parallel phase: black rows
//     y_b = inv(D_b') (d_b - sum_k L_bk d_k), then red rows y_r = inv(D_r) (d_r - sum_b A_rb y_b).
//   * On 3D grids whose dimensions are multiples of 4 the ILU(0) runs in the box-8-colour order
//     instead (ewg_box8.cuh): the solve then works in that storage order (the Jacobian is copied
//     into it once per preconditioner setup, the right-hand side and the update at the ends of a
//     solve), eight parallel colour phases per sweep, a third fewer iterations on the lens problem.
//   * FP32 instances of the same kernels run the inner solve of the mixed-precision mode.
#include <cstdio>
#include <cstring>

#include "ewg_box8.cuh"

namespace ewg {

// The BiCGStab kernels with grid reductions run on a fixed grid of kRedBlocksPerSM blocks per SM
// (deterministic partial sums); they are compiled to fit that many resident blocks, so the grid
// runs in one wave.
constexpr int kRedBlocksPerSM = 4;


// ---- deterministic grid reduction -----------------------------------------------------------

template <int NS, int NM>
__device__ __forceinline__ bool grid_reduce(double (&v)[NS + NM], double* partials, unsigned* counter,
                                            double (&out)[NS + NM]) {
    constexpr int NV = NS + NM;
    __shared__ double sh[NV][kSolBlock / 32];
    __shared__ int amLast;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_xor_sync(0xffffffffu, v[k], o);
            v[k] = k < NS ? v[k] + u : fmax(v[k], u);
        }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; ++k) {
            double a = sh[k][0];
            for (int w = 1; w < nw; ++w) a = k < NS ? a + sh[k][w] : fmax(a, sh[k][w]);
            partials[(size_t)blockIdx.x * NV + k] = a;
        }
        __threadfence();
        amLast = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!amLast) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double u = __ldcg(&partials[(size_t)b * NV + k]);
            acc[k] = k < NS ? acc[k] + u : fmax(acc[k], u);
        }
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            double u = __shfl_xor_sync(0xffffffffu, acc[k], o);
            acc[k] = k < NS ? acc[k] + u : fmax(acc[k], u);
        }
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k][warp] = acc[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; ++k) {
            double a = sh[k][0];
            for (int w = 1; w < nw; ++w) a = k < NS ? a + sh[k][w] : fmax(a, sh[k][w]);
            out[k] = a;
        }
        *counter = 0u;
    }
    return true;
}


// ---- preconditioner setup -------------------------------------------------------------------

// colour 0 (red) rows and, for block Jacobi, all rows: Dinv = inv(A_ii)
template <typename TM>
__global__ void k_diag_inverse(const __grid_constant__ Phys P, const TM* __restrict__ A, TM* __restrict__ Dinv,
                               int64_t count, int* bad) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < count;
         s += (int64_t)gridDim.x * blockDim.x)
        if (!diag_inverse_row(P.N, A, Dinv, s)) atomicOr(bad, 1);
}

// black rows: L_bk = A_bk inv(D_k) in ascending column order, D_b' = A_bb - sum L_bk A_kb
template <typename TM>
__global__ void k_ilu_black_factor(const __grid_constant__ Phys P, const TM* __restrict__ A, TM* __restrict__ Dinv,
                                   TM* __restrict__ L, int* bad) {
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < P.Nh;
         h += (int64_t)gridDim.x * blockDim.x)
        if (!ilu_black_factor_row(P, A, Dinv, L, h)) atomicOr(bad, 1);
}

// ---- preconditioner application -----------------------------------------------------------

template <typename TM, typename TV>
__global__ void __launch_bounds__(kSolBlock) k_ilu_black_apply(const __grid_constant__ Phys P, const TM* __restrict__ Dinv,
                                                                const TM* __restrict__ L,
                                                                const typename V2T<TV>::type* __restrict__ d,
                                                                typename V2T<TV>::type* __restrict__ y,
                                                                const int* __restrict__ status, double w) {
    pdl_enter();
    if (status && *status != ST_RUNNING) return;
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < P.Nh;
         h += (int64_t)gridDim.x * blockDim.x)
        ilu_black_apply_row<TM, TV>(P, Dinv, L, d, y, w, h);
}

template <typename TM, typename TV>
__global__ void __launch_bounds__(kSolBlock) k_ilu_red_apply(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                              const TM* __restrict__ Dinv,
                                                              const typename V2T<TV>::type* __restrict__ d,
                                                              typename V2T<TV>::type* __restrict__ y,
                                                              const int* __restrict__ status, double w) {
    pdl_enter();
    if (status && *status != ST_RUNNING) return;
    const double winv = 1.0 / w;
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < P.Nh;
         h += (int64_t)gridDim.x * blockDim.x)
        ilu_red_apply_row<TM, TV>(P, A, Dinv, d, y, w, winv, h);
}

template <typename TM, typename TV>
__global__ void __launch_bounds__(kSolBlock) k_jacobi_apply(const __grid_constant__ Phys P, const TM* __restrict__ Dinv,
                                                             const typename V2T<TV>::type* __restrict__ d,
                                                             typename V2T<TV>::type* __restrict__ y,
                                                             const int* __restrict__ status, double w) {
    pdl_enter();
    if (status && *status != ST_RUNNING) return;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        auto ds = d[s];
        const double r0 = (double)ds.x, r1 = (double)ds.y;
        double Di[4];
        load_block(Dinv, P.N, 0, s, Di);
        typename V2T<TV>::type out;
        out.x = (TV)(w * (Di[0] * r0 + Di[1] * r1));
        out.y = (TV)(w * (Di[2] * r0 + Di[3] * r1));
        y[s] = out;
    }
}

// ---- SpMV ----------------------------------------------------------------------------------

template <typename TM, typename TV>
__global__ void __launch_bounds__(kSolBlock) k_spmv(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                     const typename V2T<TV>::type* __restrict__ x,
                                                     typename V2T<TV>::type* __restrict__ y) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row<TM, TV>(P, A, x, s, a0, a1);
        typename V2T<TV>::type o;
        o.x = (TV)a0; o.y = (TV)a1;
        y[s] = o;
    }
}

// ---- BiCGStab kernels ------------------------------------------------------------------------

// Where the SpMV kernels find their matrix row: MODE 0 the split order, 1 box-8 order, 2 box-8
// order for a vector the box-8 ILU(0) just produced (x = relax M^-1 d with the sweeps'
// intermediate in W and E = A_cc - D': the later neighbours' blocks are not read).
struct SpmvExtra {
    const void* E;
    const void* W;
    double relax;
};

template <typename TM, typename TV, int MODE>
__device__ __forceinline__ void spmv_row_any(const Phys& P, const TM* __restrict__ A,
                                             const typename V2T<TV>::type* __restrict__ x, int64_t s,
                                             const SpmvExtra& ex, double& a0, double& a1) {
    if (MODE == 2)
        spmv_row_b8_precond<TM, TV>(P, A, (const TM*)ex.E, (const typename V2T<TV>::type*)ex.W, ex.relax, x, s, a0, a1);
    else if (MODE == 1)
        spmv_row_b8<TM, TV>(P, A, x, s, a0, a1);
    else
        spmv_row<TM, TV>(P, A, x, s, a0, a1);
}

template <typename TV>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_init(const __grid_constant__ Phys P,
                                                          const typename V2T<TV>::type* __restrict__ b,
                                                          typename V2T<TV>::type* __restrict__ x,
                                                          typename V2T<TV>::type* __restrict__ r,
                                                          typename V2T<TV>::type* __restrict__ r0,
                                                          typename V2T<TV>::type* __restrict__ v,
                                                          typename V2T<TV>::type* __restrict__ p,
                                                          BiState* st, double* partials, unsigned* counter) {
    double red[2] = {0.0, 0.0};  // sum b.b, max |b|
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        auto bs = b[s];
        typename V2T<TV>::type z;
        z.x = (TV)0; z.y = (TV)0;
        x[s] = z; v[s] = z; p[s] = z;
        r[s] = bs; r0[s] = bs;
        const double b0 = (double)bs.x, b1 = (double)bs.y;
        red[0] += b0 * b0 + b1 * b1;
        red[1] = fmax(red[1], fmax(absn(b0), absn(b1)));
    }
    double out[2];
    if (grid_reduce<1, 1>(red, partials, counter, out) && threadIdx.x == 0) {
        // CombinedCriterion::setInitial
        st->resErr = fmax(out[1], DBL_MIN * 1e10);
        st->initResErr = st->resErr;
        st->lastResErr = st->resErr;
        st->stagnates = 0;
        st->iter = 0;
        st->restarts = 0;
        st->restartPending = 0;
        st->rho = 1.0; st->alpha = 1.0; st->omega = 1.0;
        st->r0r0 = out[0];
        st->status = ST_RUNNING;
        double rel = st->resErr / fmax(1e-20, st->initResErr);
        if (rel <= st->relTol || st->resErr <= st->absTol) { st->status = ST_CONVERGED; return; }
        iteration_top(st, out[0], out[0]);
    }
}

// p = r + (-beta) (omega v - p); on a restart r0hat = r, v = p = 0 first
template <typename TV>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_p(const __grid_constant__ Phys P,
                                                       const typename V2T<TV>::type* __restrict__ r,
                                                       typename V2T<TV>::type* __restrict__ r0,
                                                       typename V2T<TV>::type* __restrict__ v,
                                                       typename V2T<TV>::type* __restrict__ p,
                                                       const BiState* __restrict__ st) {
    pdl_enter();
    if (st->status != ST_RUNNING) return;
    const bool restart = st->restartPending != 0;
    const double beta = st->beta, omega = st->omega;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        auto rs = r[s];
        typename V2T<TV>::type vs = v[s], ps = p[s];
        if (restart) {
            r0[s] = rs;
            vs.x = (TV)0; vs.y = (TV)0;
            ps = vs;
            v[s] = vs;
        }
        double t0 = (double)vs.x * omega, t1 = (double)vs.y * omega;
        t0 -= (double)ps.x; t1 -= (double)ps.y;
        t0 *= -beta; t1 *= -beta;
        typename V2T<TV>::type o;
        o.x = (TV)((double)rs.x + t0);
        o.y = (TV)((double)rs.y + t1);
        p[s] = o;
    }
}

// v = A y; alpha = rho_i / (r0hat . v)
template <typename TM, typename TV, int MODE>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_spmv_alpha(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                                const typename V2T<TV>::type* __restrict__ y,
                                                                const typename V2T<TV>::type* __restrict__ r0,
                                                                typename V2T<TV>::type* __restrict__ v,
                                                                BiState* st, double* partials, unsigned* counter,
                                                                const SpmvExtra ex) {
    pdl_enter();
    if (st->status != ST_RUNNING) return;
    double red[1] = {0.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row_any<TM, TV, MODE>(P, A, y, s, ex, a0, a1);
        typename V2T<TV>::type o;
        o.x = (TV)a0; o.y = (TV)a1;
        v[s] = o;
        auto rh = r0[s];
        red[0] += (double)rh.x * (double)o.x + (double)rh.y * (double)o.y;
    }
    double out[1];
    if (grid_reduce<1, 0>(red, partials, counter, out) && threadIdx.x == 0) {
        const double breakdownEps = DBL_MIN * 1e10;
        st->restartPending = 0;
        double denom = out[0];
        if (fabs(denom) <= breakdownEps) { st->status = ST_BREAKDOWN; return; }
        st->alpha = st->rho_i / denom;
        if (fabs(st->alpha) <= breakdownEps) st->status = ST_BREAKDOWN;
    }
}

// h = x + alpha y (in x), s = r - alpha v (in r); criterion on s with y as change indicator
template <typename TV>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_hs(const __grid_constant__ Phys P,
                                                        typename V2T<TV>::type* __restrict__ x,
                                                        const typename V2T<TV>::type* __restrict__ y,
                                                        typename V2T<TV>::type* __restrict__ r,
                                                        const typename V2T<TV>::type* __restrict__ v,
                                                        BiState* st, double* partials, unsigned* counter) {
    pdl_enter();
    if (st->status != ST_RUNNING) return;
    const double alpha = st->alpha;
    double red[2] = {0.0, 0.0};  // max |s|, any y != 0
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        auto ys = y[s], xs = x[s], rs = r[s], vs = v[s];
        typename V2T<TV>::type hx, sx;
        hx.x = (TV)((double)ys.x * alpha + (double)xs.x);
        hx.y = (TV)((double)ys.y * alpha + (double)xs.y);
        sx.x = (TV)((double)rs.x - (double)vs.x * alpha);
        sx.y = (TV)((double)rs.y - (double)vs.y * alpha);
        x[s] = hx;
        r[s] = sx;
        red[0] = fmax(red[0], fmax(absn((double)sx.x), absn((double)sx.y)));
        if (ys.x != (TV)0 || ys.y != (TV)0) red[1] = 1.0;
    }
    double out[2];
    if (grid_reduce<0, 2>(red, partials, counter, out) && threadIdx.x == 0) {
        st->lastResErr = st->resErr;
        st->resErr = out[0];
        st->stagnates = out[1] == 0.0;
        criterion_check(st);
    }
}

// t = A z; omega = (t . s) / (t . t)
template <typename TM, typename TV, int MODE>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_spmv_omega(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                                const typename V2T<TV>::type* __restrict__ z,
                                                                const typename V2T<TV>::type* __restrict__ sres,
                                                                typename V2T<TV>::type* __restrict__ t,
                                                                BiState* st, double* partials, unsigned* counter,
                                                                const SpmvExtra ex) {
    pdl_enter();
    if (st->status != ST_RUNNING) return;
    double red[2] = {0.0, 0.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row_any<TM, TV, MODE>(P, A, z, s, ex, a0, a1);
        typename V2T<TV>::type o;
        o.x = (TV)a0; o.y = (TV)a1;
        t[s] = o;
        auto ss = sres[s];
        const double t0 = (double)o.x, t1 = (double)o.y;
        red[0] += t0 * t0 + t1 * t1;
        red[1] += t0 * (double)ss.x + t1 * (double)ss.y;
    }
    double out[2];
    if (grid_reduce<2, 0>(red, partials, counter, out) && threadIdx.x == 0) {
        const double breakdownEps = DBL_MIN * 1e10;
        if (fabs(out[0]) <= breakdownEps) { st->status = ST_BREAKDOWN; return; }
        st->omega = out[1] / out[0];
        if (fabs(st->omega) <= breakdownEps) st->status = ST_BREAKDOWN;
    }
}

// x += omega z; criterion on r (still s) with z as change indicator; r += -omega t;
// then the next iteration's r0hat . r and r . r
template <typename TV>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_xr(const __grid_constant__ Phys P,
                                                        typename V2T<TV>::type* __restrict__ x,
                                                        const typename V2T<TV>::type* __restrict__ z,
                                                        typename V2T<TV>::type* __restrict__ r,
                                                        const typename V2T<TV>::type* __restrict__ t,
                                                        const typename V2T<TV>::type* __restrict__ r0,
                                                        BiState* st, double* partials, unsigned* counter) {
    pdl_enter();
    if (st->status != ST_RUNNING) return;
    const double omega = st->omega;
    double red[4] = {0.0, 0.0, 0.0, 0.0};  // sum r0.r', sum r'.r', max |s|, any z != 0
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        auto xs = x[s], zs = z[s], rs = r[s], ts = t[s], rh = r0[s];
        typename V2T<TV>::type xn, rn;
        xn.x = (TV)((double)xs.x + omega * (double)zs.x);
        xn.y = (TV)((double)xs.y + omega * (double)zs.y);
        x[s] = xn;
        red[2] = fmax(red[2], fmax(absn((double)rs.x), absn((double)rs.y)));
        if (zs.x != (TV)0 || zs.y != (TV)0) red[3] = 1.0;
        rn.x = (TV)((double)rs.x + (-omega) * (double)ts.x);
        rn.y = (TV)((double)rs.y + (-omega) * (double)ts.y);
        r[s] = rn;
        const double r0v = (double)rn.x, r1v = (double)rn.y;
        red[0] += (double)rh.x * r0v + (double)rh.y * r1v;
        red[1] += r0v * r0v + r1v * r1v;
    }
    double out[4];
    if (grid_reduce<2, 2>(red, partials, counter, out) && threadIdx.x == 0) {
        st->lastResErr = st->resErr;
        st->resErr = out[2];
        st->stagnates = out[3] == 0.0;
        criterion_check(st);
        if (st->status != ST_RUNNING) return;
        st->iter += 1;
        iteration_top(st, out[0], out[1]);
    }
}

// Residual replacement after convergence: r = r0hat = b - A x with max-norm and r . r. If the
// true residual misses the criterion by more than 10x the iteration resumes from x.
template <typename TM, typename TV, int MODE>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_bicg_true_residual(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                                   const typename V2T<TV>::type* __restrict__ b,
                                                                   const typename V2T<TV>::type* __restrict__ x,
                                                                   typename V2T<TV>::type* __restrict__ r,
                                                                   typename V2T<TV>::type* __restrict__ r0,
                                                                   typename V2T<TV>::type* __restrict__ v,
                                                                   typename V2T<TV>::type* __restrict__ p,
                                                                   BiState* st, double* partials, unsigned* counter) {
    if (st->status != ST_CONVERGED) return;
    double red[2] = {0.0, 0.0};  // sum r.r, max |r|
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row_any<TM, TV, MODE>(P, A, x, s, SpmvExtra{nullptr, nullptr, 1.0}, a0, a1);
        auto bs = b[s];
        typename V2T<TV>::type o, z;
        o.x = (TV)((double)bs.x - a0);
        o.y = (TV)((double)bs.y - a1);
        z.x = (TV)0; z.y = (TV)0;
        r[s] = o; r0[s] = o; v[s] = z; p[s] = z;
        red[0] += (double)o.x * (double)o.x + (double)o.y * (double)o.y;
        red[1] = fmax(red[1], fmax(absn((double)o.x), absn((double)o.y)));
    }
    double out[2];
    if (grid_reduce<1, 1>(red, partials, counter, out) && threadIdx.x == 0) {
        const double err = out[1];
        if (err / fmax(1e-20, st->initResErr) <= 10 * st->relTol || err <= 10 * st->absTol) return;
        st->replacements += 1;
        st->restarts += 1;
        st->status = ST_RUNNING;
        st->lastResErr = st->resErr;
        st->resErr = err;
        st->stagnates = 0;
        st->restartPending = 0;
        st->rho = 1.0; st->alpha = 1.0; st->omega = 1.0;
        st->r0r0 = out[0];
        st->iter += 1;
        iteration_top(st, out[0], out[0]);
    }
}

// ---- one slab's BiCGStab iteration in a distributed solve ---------------------------------------
//
// The same fused updates as the kernels above, for dd.distributed_bicgstab: vectors are device
// vectors in the context's storage order, the scalars (alpha, omega, beta, the restart flag) come
// from a BiState in device memory that k_slab_state advances from the reductions combined over
// all slabs, and every reduction runs over the slab's owned rows -- rows [lo, hi) of each colour
// half -- and ends, deterministically, in a small device array `out`. Rows outside [lo, hi)
// (ghost planes) are updated too; the exchange overwrites them. Once the state has left RUNNING
// every kernel returns at once, so the host reads the status only every few iterations.

__device__ __forceinline__ bool owned_row(const Phys& P, int64_t s, int64_t lo, int64_t hi) {
    const int64_t h = s >= P.Nh ? s - P.Nh : s;
    return h >= lo && h < hi;
}

// p = r + beta (p - omega v); on a restart r0 = r and v = p = 0 first
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_slab_p(const __grid_constant__ Phys P, double2* __restrict__ p,
                                                       const double2* __restrict__ r, double2* __restrict__ r0,
                                                       double2* __restrict__ v, const BiState* __restrict__ st) {
    if (st->status != ST_RUNNING) return;
    const double beta = st->beta, omega = st->omega;
    const bool restart = st->restartPending != 0;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        const double2 rs = r[s];
        double2 vs = v[s], ps = p[s];
        if (restart) {
            r0[s] = rs;
            vs = make_double2(0.0, 0.0);
            ps = vs;
            v[s] = vs;
        }
        // (omega v - p)(-beta) + r, the order of k_bicg_p
        double t0 = vs.x * omega, t1 = vs.y * omega;
        t0 -= ps.x; t1 -= ps.y;
        t0 *= -beta; t1 *= -beta;
        p[s] = make_double2(rs.x + t0, rs.y + t1);
    }
}

// y = J x; out[0] = sum over owned rows of w . y
template <int MODE>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_slab_spmv_dot(const __grid_constant__ Phys P, const double* __restrict__ A,
                                                              const double2* __restrict__ x, double2* __restrict__ y,
                                                              const double2* __restrict__ w, int64_t lo, int64_t hi,
                                                              const BiState* __restrict__ st, double* partials,
                                                              unsigned* counter, double* out) {
    if (st && st->status != ST_RUNNING) return;
    double red[1] = {0.0};
    const SpmvExtra ex{nullptr, nullptr, 1.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row_any<double, double, MODE>(P, A, x, s, ex, a0, a1);
        y[s] = make_double2(a0, a1);
        if (owned_row(P, s, lo, hi)) {
            const double2 ws = w[s];
            red[0] += ws.x * a0 + ws.y * a1;
        }
    }
    double o[1];
    if (grid_reduce<1, 0>(red, partials, counter, o) && threadIdx.x == 0) out[0] = o[0];
}

// y = J z; out = {t.t, t.s} over owned rows (t = y)
template <int MODE>
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_slab_spmv_dot2(const __grid_constant__ Phys P, const double* __restrict__ A,
                                                               const double2* __restrict__ z, double2* __restrict__ t,
                                                               const double2* __restrict__ sres, int64_t lo, int64_t hi,
                                                               const BiState* __restrict__ st, double* partials,
                                                               unsigned* counter, double* out) {
    if (st && st->status != ST_RUNNING) return;
    double red[2] = {0.0, 0.0};
    const SpmvExtra ex{nullptr, nullptr, 1.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row_any<double, double, MODE>(P, A, z, s, ex, a0, a1);
        t[s] = make_double2(a0, a1);
        if (owned_row(P, s, lo, hi)) {
            const double2 ss = sres[s];
            red[0] += a0 * a0 + a1 * a1;
            red[1] += a0 * ss.x + a1 * ss.y;
        }
    }
    double o[2];
    if (grid_reduce<2, 0>(red, partials, counter, o) && threadIdx.x == 0) { out[0] = o[0]; out[1] = o[1]; }
}

// x += alpha y (h); r -= alpha v (s); out = {max |s|, max |y|} over owned rows
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_slab_hs(const __grid_constant__ Phys P, double2* __restrict__ x,
                                                        const double2* __restrict__ y, double2* __restrict__ r,
                                                        const double2* __restrict__ v, int64_t lo, int64_t hi,
                                                        const BiState* __restrict__ st, double* partials,
                                                        unsigned* counter, double* out) {
    if (st->status != ST_RUNNING) return;
    const double alpha = st->alpha;
    double red[2] = {0.0, 0.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        const double2 ys = y[s], vs = v[s];
        double2 xs = x[s], rs = r[s];
        xs.x = ys.x * alpha + xs.x; xs.y = ys.y * alpha + xs.y;
        rs.x = rs.x - vs.x * alpha; rs.y = rs.y - vs.y * alpha;
        x[s] = xs;
        r[s] = rs;
        if (owned_row(P, s, lo, hi)) {
            red[0] = fmax(red[0], fmax(absn(rs.x), absn(rs.y)));
            red[1] = fmax(red[1], fmax(absn(ys.x), absn(ys.y)));
        }
    }
    double o[2];
    if (grid_reduce<0, 2>(red, partials, counter, o) && threadIdx.x == 0) { out[0] = o[0]; out[1] = o[1]; }
}

// x += omega z; then {max |s|, max |z|} over owned rows (r still holds s); r += -omega t;
// out = {r0 . r, r . r, max |s|, max |z|}
__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_slab_xr(const __grid_constant__ Phys P, double2* __restrict__ x,
                                                        const double2* __restrict__ z, double2* __restrict__ r,
                                                        const double2* __restrict__ t, const double2* __restrict__ r0,
                                                        int64_t lo, int64_t hi, const BiState* __restrict__ st,
                                                        double* partials, unsigned* counter, double* out) {
    if (st->status != ST_RUNNING) return;
    const double omega = st->omega;
    double red[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        const double2 zs = z[s], ts = t[s];
        double2 xs = x[s], rs = r[s];
        xs.x = xs.x + omega * zs.x; xs.y = xs.y + omega * zs.y;
        x[s] = xs;
        const bool own = owned_row(P, s, lo, hi);
        if (own) {
            red[2] = fmax(red[2], fmax(absn(rs.x), absn(rs.y)));
            red[3] = fmax(red[3], fmax(absn(zs.x), absn(zs.y)));
        }
        rs.x = rs.x + (-omega) * ts.x; rs.y = rs.y + (-omega) * ts.y;
        r[s] = rs;
        if (own) {
            const double2 rh = r0[s];
            red[0] += rh.x * rs.x + rh.y * rs.y;
            red[1] += rs.x * rs.x + rs.y * rs.y;
        }
    }
    double o[4];
    if (grid_reduce<2, 2>(red, partials, counter, o) && threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) out[k] = o[k];
}

// One scalar step of the distributed BiCGStab on the reductions combined over all slabs, the
// decisions the single-domain kernels take in their last block (BiCGStabSolver::apply,
// CombinedCriterion, bicgstabsolver.hh:191-322, combinedcriterion.hh:112-205).
//   0 start  red = {b.b, max|b|}            setInitial, then the top of the first iteration
//   1 alpha  red = {r0.v}                    alpha = rho_i / r0.v, breakdown tests
//   2 half   red = {t.t, t.s, max|s|, max|y|}  criterion on s (y all zero: stagnation), omega
//   3 full   red = {r0.r, r.r, max|s|, max|z|} criterion on s, next iteration's top
//   4 true   red = {r.r, max|r|}             after convergence, on r = b - J x: resume from x when
//                                             the true residual misses the criterion by 10x
__global__ void k_slab_state(int stage, BiState* st, const double* __restrict__ red, double relTol, double absTol,
                             double maxRes, int maxIter, int restartOnBreakdown) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double breakdownEps = DBL_MIN * 1e10;
    if (stage == 0) {
        memset(st, 0, sizeof(BiState));
        st->relTol = relTol; st->absTol = absTol; st->maxRes = maxRes; st->maxIter = maxIter;
        st->restartOnBreakdown = restartOnBreakdown;
        st->resErr = fmax(red[1], breakdownEps);
        st->initResErr = st->resErr;
        st->lastResErr = st->resErr;
        st->rho = 1.0; st->alpha = 1.0; st->omega = 1.0;
        st->r0r0 = red[0];
        st->status = ST_RUNNING;
        if (st->resErr / fmax(1e-20, st->initResErr) <= relTol || st->resErr <= absTol) { st->status = ST_CONVERGED; return; }
        iteration_top(st, red[0], red[0]);
        return;
    }
    if (stage == 4) {
        if (st->status != ST_CONVERGED) return;
        const double err = red[1];
        if (err / fmax(1e-20, st->initResErr) <= 10 * st->relTol || err <= 10 * st->absTol) return;
        st->replacements += 1;
        st->restarts += 1;
        st->status = ST_RUNNING;
        st->lastResErr = st->resErr;
        st->resErr = err;
        st->stagnates = 0;
        st->restartPending = 0;
        st->rho = 1.0; st->alpha = 1.0; st->omega = 1.0;
        st->r0r0 = red[0];
        st->iter += 1;
        iteration_top(st, red[0], red[0]);
        return;
    }
    if (st->status != ST_RUNNING) return;
    if (stage == 1) {
        st->restartPending = 0;
        const double denom = red[0];
        if (fabs(denom) <= breakdownEps) { st->status = ST_BREAKDOWN; return; }
        st->alpha = st->rho_i / denom;
        if (fabs(st->alpha) <= breakdownEps) st->status = ST_BREAKDOWN;
    } else if (stage == 2) {
        st->lastResErr = st->resErr;
        st->resErr = red[2];
        st->stagnates = red[3] == 0.0;
        criterion_check(st);
        if (st->status != ST_RUNNING) return;
        if (fabs(red[0]) <= breakdownEps) { st->status = ST_BREAKDOWN; return; }
        st->omega = red[1] / red[0];
        if (fabs(st->omega) <= breakdownEps) st->status = ST_BREAKDOWN;
    } else if (stage == 3) {
        st->lastResErr = st->resErr;
        st->resErr = red[2];
        st->stagnates = red[3] == 0.0;
        criterion_check(st);
        if (st->status != ST_RUNNING) return;
        st->iter += 1;
        iteration_top(st, red[0], red[1]);
    }
}

// ---- mixed precision: defect correction ----------------------------------------------------

__global__ void k_to_float(const __grid_constant__ Phys P, const double2* __restrict__ a, float2* __restrict__ b) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double2 v = a[s];
        b[s] = make_float2((float)v.x, (float)v.y);
    }
}

// x64 += dx32; r64 = b - A32 x64 (FP64 arithmetic); max |r64| into *maxOut (ordered bits)
__global__ void k_defect_accumulate(const __grid_constant__ Phys P, double2* __restrict__ x64, const float2* __restrict__ dx32) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        float2 d = dx32[s];
        double2 x = x64[s];
        x.x += (double)d.x;
        x.y += (double)d.y;
        x64[s] = x;
    }
}

__global__ void __launch_bounds__(kSolBlock, kRedBlocksPerSM) k_defect_residual(const __grid_constant__ Phys P, const float* __restrict__ A,
                                                                const double2* __restrict__ b,
                                                                const double2* __restrict__ x64,
                                                                double2* __restrict__ r64, double* partials,
                                                                unsigned* counter, double* maxOut) {
    double red[1] = {0.0};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double a0, a1;
        spmv_row<float, double>(P, A, x64, s, a0, a1);
        double2 bs = b[s];
        double2 o = make_double2(bs.x - a0, bs.y - a1);
        r64[s] = o;
        red[0] = fmax(red[0], fmax(absn(o.x), absn(o.y)));
    }
    double out[1];
    if (grid_reduce<0, 1>(red, partials, counter, out) && threadIdx.x == 0) *maxOut = out[0];
}

// ---- Newton update --------------------------------------------------------------------------

__global__ void k_newton_update(const __grid_constant__ Phys P, double2* __restrict__ x, const double2* __restrict__ dx, int* bad) {
    int b = 0;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        double2 d = dx[s];
        if (!isfinite(d.x) || !isfinite(d.y)) b = 1;
        double2 v = x[s];
        v.x -= d.x;
        v.y -= d.y;
        x[s] = v;
    }
    if (b) atomicOr(bad, 1);
}

// ---- host side ------------------------------------------------------------------------------

// Workspace for one precision: Krylov vectors, ILU factors, reduction scratch.
template <typename T>
struct KrylovWs {
    using V = typename V2T<T>::type;
    V *x = nullptr, *r = nullptr, *r0 = nullptr, *v = nullptr, *p = nullptr, *y = nullptr, *z = nullptr, *b = nullptr;
    T* Dinv = nullptr;   // 4 planes x N
    T* L = nullptr;      // (2*dim*4) planes x Nh (black rows)
    // box-8-colour ILU(0) (allocated on first use): the matrix in box-8 order, its L factors
    // (6 bands x 4 planes x N; only the earlier neighbour of each face is written), the inverted
    // pivots, and two vectors for preconditioner calls on split-order vectors
    T* A8 = nullptr;
    T* L8 = nullptr;
    T* Dinv8 = nullptr;
    T* E8 = nullptr;     // A_cc - D' per cell (4 planes x N)
    V* W = nullptr;      // forward-sweep intermediate of the last preconditioner application
    V *t0 = nullptr, *t1 = nullptr;
};

struct SolverWs {
    KrylovWs<double> d;
    KrylovWs<float> f;
    double2* x64 = nullptr;   // mixed: accumulated solution
    double2* r64 = nullptr;   // mixed: FP64 defect
    double* partials = nullptr;
    unsigned* counter = nullptr;
    BiState* st = nullptr;
    int* flags = nullptr;     // [0] singular block
    double* dmax = nullptr;
    BiState* h_st = nullptr;  // pinned mirror
    int gridRed = 0;
    bool haveF = false;
};

template <typename T>
static cudaError_t alloc_ws(KrylovWs<T>& w, const Phys& P) {
    using V = typename V2T<T>::type;
    cudaError_t e;
    V** vs[] = {&w.x, &w.r, &w.r0, &w.v, &w.p, &w.y, &w.z, &w.b};
    for (V** q : vs)
        if ((e = cudaMalloc(q, sizeof(V) * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.Dinv, sizeof(T) * 4 * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.L, sizeof(T) * 4 * 2 * P.dim * P.Nh)) != cudaSuccess) return e;
    return cudaSuccess;
}
template <typename T>
static cudaError_t alloc_b8(KrylovWs<T>& w, const Phys& P) {
    using V = typename V2T<T>::type;
    cudaError_t e;
    if (w.A8) return cudaSuccess;
    if ((e = cudaMalloc(&w.A8, sizeof(T) * 4 * 7 * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.L8, sizeof(T) * 4 * 6 * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.Dinv8, sizeof(T) * 4 * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.E8, sizeof(T) * 4 * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.W, sizeof(V) * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.t0, sizeof(V) * P.N)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.t1, sizeof(V) * P.N)) != cudaSuccess) return e;
    return cudaSuccess;
}
template <typename T>
static void free_ws(KrylovWs<T>& w) {
    void* b8[] = {w.A8, w.L8, w.Dinv8, w.E8, w.W, w.t0, w.t1};
    for (void* q : b8) if (q) cudaFree(q);
    void* ps[] = {w.x, w.r, w.r0, w.v, w.p, w.y, w.z, w.b, w.Dinv, w.L};
    for (void* q : ps) if (q) cudaFree(q);
    w = KrylovWs<T>();
}

static SolverWs* ws_of(ewg_ctx* ctx) { return (SolverWs*)ctx->sv; }

static ewg_status ensure_ws(ewg_ctx* ctx, bool needFloat) {
    cudaError_t e;
    if (!ctx->sv) {
        SolverWs* w = new SolverWs();
        ctx->sv = w;
        if ((e = alloc_ws(w->d, ctx->P)) != cudaSuccess) return cuda_fail(ctx, e, "alloc solver vectors");
        w->gridRed = ctx->numSMs * kRedBlocksPerSM;
        if ((e = cudaMalloc(&w->partials, sizeof(double) * kMaxRed * w->gridRed * 2)) != cudaSuccess) return cuda_fail(ctx, e, "alloc partials");
        if ((e = cudaMalloc(&w->counter, sizeof(unsigned) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "alloc counter");
        if ((e = cudaMemsetAsync(w->counter, 0, sizeof(unsigned) * 4, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "memset counter");
        if ((e = cudaMalloc(&w->st, sizeof(BiState))) != cudaSuccess) return cuda_fail(ctx, e, "alloc state");
        if ((e = cudaMalloc(&w->flags, sizeof(int) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "alloc flags");
        if ((e = cudaMalloc(&w->dmax, sizeof(double) * 2)) != cudaSuccess) return cuda_fail(ctx, e, "alloc dmax");
        if ((e = cudaMallocHost(&w->h_st, sizeof(BiState))) != cudaSuccess) return cuda_fail(ctx, e, "alloc pinned state");
    }
    SolverWs* w = ws_of(ctx);
    if (needFloat && !w->haveF) {
        if ((e = alloc_ws(w->f, ctx->P)) != cudaSuccess) return cuda_fail(ctx, e, "alloc fp32 solver vectors");
        if ((e = cudaMalloc(&w->x64, sizeof(double2) * ctx->P.N)) != cudaSuccess) return cuda_fail(ctx, e, "alloc x64");
        if ((e = cudaMalloc(&w->r64, sizeof(double2) * ctx->P.N)) != cudaSuccess) return cuda_fail(ctx, e, "alloc r64");
        w->haveF = true;
    }
    return EWG_OK;
}

void solver_free(ewg_ctx* ctx) {
    SolverWs* w = ws_of(ctx);
    if (!w) return;
    free_ws(w->d);
    free_ws(w->f);
    void* ps[] = {w->x64, w->r64, w->partials, w->counter, w->st, w->flags, w->dmax};
    for (void* q : ps) if (q) cudaFree(q);
    if (w->h_st) cudaFreeHost(w->h_st);
    delete w;
    ctx->sv = nullptr;
}

template <typename T>
static const T* jac_of(ewg_ctx* ctx);
template <> const double* jac_of<double>(ewg_ctx* ctx) { return ctx->J; }
template <> const float* jac_of<float>(ewg_ctx* ctx) { return ctx->J32; }

template <typename T>
static ewg_status setup_precond(ewg_ctx* ctx, KrylovWs<T>& w, int kind) {
    const Phys& P = ctx->P;
    SolverWs* sw = ws_of(ctx);
    cudaError_t e;
    if ((e = cudaMemsetAsync(sw->flags, 0, sizeof(int), ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "memset flags");
    const T* A = jac_of<T>(ctx);
    if (kind == EWG_PRECOND_JACOBI) {
        int g = grid_size_for(ctx, (const void*)k_diag_inverse<T>, kSolBlock);
        EWG_LAUNCH(ctx, K_DIAG_INVERSE, k_diag_inverse<T>, g, kSolBlock, P, A, w.Dinv, P.N, sw->flags);
    } else {
        int g = grid_size_for(ctx, (const void*)k_diag_inverse<T>, kSolBlock);
        EWG_LAUNCH(ctx, K_DIAG_INVERSE, k_diag_inverse<T>, g, kSolBlock, P, A, w.Dinv, P.Nh, sw->flags);
        int g2 = grid_size_for(ctx, (const void*)k_ilu_black_factor<T>, kSolBlock);
        EWG_LAUNCH(ctx, K_ILU_BLACK_FACTOR, k_ilu_black_factor<T>, g2, kSolBlock, P, A, w.Dinv, w.L, sw->flags);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "preconditioner setup");
    int bad = 0;
    if ((e = cudaMemcpyAsync(&bad, sw->flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "read flags");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync precond");
    if (bad) {
        ctx->err = "preconditioner: singular 2x2 diagonal block";
        return EWG_ERR_BREAKDOWN;
    }
    return EWG_OK;
}

template <typename T>
static void launch_precond(ewg_ctx* ctx, KrylovWs<T>& w, int kind, double relax,
                           const typename V2T<T>::type* d, typename V2T<T>::type* y, const int* status) {
    const Phys& P = ctx->P;
    const T* A = jac_of<T>(ctx);
    if (kind == EWG_PRECOND_JACOBI) {
        int g = grid_size_for(ctx, (const void*)k_jacobi_apply<T, T>, kSolBlock);
        {
            auto kfn = k_jacobi_apply<T, T>;
            EWG_LAUNCH_PDL(ctx, K_JACOBI_APPLY, kfn, g, kSolBlock, P, w.Dinv, d, y, status, relax);
        }
    } else {
        int g = grid_size_for(ctx, (const void*)k_ilu_black_apply<T, T>, kSolBlock);
        {
            auto kfn = k_ilu_black_apply<T, T>;
            EWG_LAUNCH_PDL(ctx, K_ILU_BLACK_APPLY, kfn, g, kSolBlock, P, w.Dinv, w.L, d, y, status, relax);
        }
        int g2 = grid_size_for(ctx, (const void*)k_ilu_red_apply<T, T>, kSolBlock);
        {
            auto kfn = k_ilu_red_apply<T, T>;
            EWG_LAUNCH_PDL(ctx, K_ILU_RED_APPLY, kfn, g2, kSolBlock, P, A, w.Dinv, d, y, status, relax);
        }
    }
}

// Does this solve run its ILU(0) in the box-8-colour order?
static bool use_b8(const ewg_ctx* ctx, const ewg_solve_opts* o) {
    if (o->precond != EWG_PRECOND_ILU0) return false;
    if (o->ilu_ordering == EWG_ILU_ORDER_REDBLACK) return false;
    return ctx->P.b8ok != 0;  // AUTO or BOX8 (BOX8 on an unsuitable grid is rejected by the caller)
}

static ewg_status check_ordering(ewg_ctx* ctx, const ewg_solve_opts* o) {
    if (o->ilu_ordering < EWG_ILU_ORDER_AUTO || o->ilu_ordering > EWG_ILU_ORDER_BOX8) {
        ctx->err = "unknown ilu_ordering";
        return EWG_ERR_INVALID;
    }
    if (o->ilu_ordering == EWG_ILU_ORDER_BOX8 && o->precond == EWG_PRECOND_ILU0 && !ctx->P.b8ok) {
        ctx->err = "ilu_ordering BOX8 needs a 3D grid with nx, ny and nz multiples of 4";
        return EWG_ERR_INVALID;
    }
    return EWG_OK;
}

// Box-8-colour ILU(0): the Jacobian copied into box-8 order, then the eight colours factorized
// one after another.
template <typename T>
static ewg_status setup_precond_b8(ewg_ctx* ctx, KrylovWs<T>& w) {
    const Phys& P = ctx->P;
    SolverWs* sw = ws_of(ctx);
    cudaError_t e;
    if ((e = alloc_b8(w, P)) != cudaSuccess) return cuda_fail(ctx, e, "alloc box-8 ILU");
    if ((e = cudaMemsetAsync(sw->flags, 0, sizeof(int), ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "memset flags");
    b8_matrix_from_split<T, T>(ctx, 28, jac_of<T>(ctx), w.A8);
    b8_factor<T>(ctx, w.A8, w.Dinv8, w.L8, w.E8, sw->flags);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "box-8 ILU setup");
    int bad = 0;
    if ((e = cudaMemcpyAsync(&bad, sw->flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "read flags");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync box-8 ILU");
    if (bad) {
        ctx->err = "preconditioner: singular 2x2 diagonal block";
        return EWG_ERR_BREAKDOWN;
    }
    return EWG_OK;
}

// y = relax * M^-1 d in box-8 order (d and y distinct); the forward intermediate stays in w.W
template <typename T>
static void launch_precond_b8(ewg_ctx* ctx, KrylovWs<T>& w, double relax, const typename V2T<T>::type* d,
                              typename V2T<T>::type* y, const int* status) {
    b8_apply<T>(ctx, w.A8, w.Dinv8, w.L8, relax, d, w.W, y, status);
}

// split order <-> box-8 order for one vector, with a precision change
template <typename TI, typename TO, bool TOB8>
static void launch_b8_vector(ewg_ctx* ctx, const typename V2T<TI>::type* in, typename V2T<TO>::type* out) {
    b8_vector<TI, TO, TOB8>(ctx, in, out);
}

// set up the preconditioner of the requested kind and order unless it is current
template <typename T>
static ewg_status ensure_precond(ewg_ctx* ctx, KrylovWs<T>& w, const ewg_solve_opts* o, int precision) {
    const int order = use_b8(ctx, o) ? EWG_ILU_ORDER_BOX8 : EWG_ILU_ORDER_REDBLACK;
    if (ctx->iluValid && ctx->iluKind == o->precond && ctx->iluPrecision == precision && ctx->iluOrder == order)
        return EWG_OK;
    ewg_status st = order == EWG_ILU_ORDER_BOX8 ? setup_precond_b8<T>(ctx, w) : setup_precond<T>(ctx, w, o->precond);
    if (st) return st;
    ctx->iluValid = true;
    ctx->iluKind = o->precond;
    ctx->iluPrecision = precision;
    ctx->iluOrder = order;
    return EWG_OK;
}

// One BiCGStab solve of A x = b for the precision T; b must already be in w.b (in box-8 order
// when the solve runs its ILU(0) in that order).
template <typename T>
static ewg_status bicgstab(ewg_ctx* ctx, KrylovWs<T>& w, const ewg_solve_opts* o, double relTol, double absTol,
                           int maxIter, int* itersOut, int* restartsOut, double* resOut, int* statusOut,
                           double* initOut = nullptr) {
    const Phys& P = ctx->P;
    SolverWs* sw = ws_of(ctx);
    const bool b8 = use_b8(ctx, o);
    const T* A = b8 ? w.A8 : jac_of<T>(ctx);
    cudaError_t e;
    BiState init;
    memset(&init, 0, sizeof(init));
    init.relTol = relTol;
    init.absTol = absTol;
    init.maxRes = o->linear_solver_max_error;
    init.maxIter = maxIter;
    init.restartOnBreakdown = o->restart_on_breakdown;
    init.verifyTrue = o->verify_true_residual;
    init.w = o->preconditioner_relaxation;
    if ((e = cudaMemcpyAsync(sw->st, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "upload state");
    const int G = sw->gridRed;
    double* part = sw->partials;
    unsigned* cnt = sw->counter;
    EWG_LAUNCH(ctx, K_BICG_INIT, k_bicg_init<T>, G, kSolBlock, P, w.b, w.x, w.r, w.r0, w.v, w.p, sw->st, part, cnt);
    // host status reads: every kernel launched after the solve has ended returns at once, so a few
    // iterations' launches past convergence cost microseconds, while a read per iteration leaves
    // the device idle for a host round trip every iteration
    int interval = o->check_interval > 0 ? o->check_interval : (P.N >= (1 << 20) ? 4 : 8);
    const int* status = &sw->st->status;
    const double relax = o->preconditioner_relaxation;
    const SpmvExtra ex{b8 ? (const void*)w.E8 : nullptr, b8 ? (const void*)w.W : nullptr, relax};
    int guard = 0;
    for (;;) {
        for (int k = 0; k < interval; ++k) {
            EWG_LAUNCH_PDL(ctx, K_BICG_P, k_bicg_p<T>, G, kSolBlock, P, w.r, w.r0, w.v, w.p, sw->st);
            if (b8) launch_precond_b8<T>(ctx, w, relax, w.p, w.y, status);
            else launch_precond<T>(ctx, w, o->precond, relax, w.p, w.y, status);
            {
                auto kfn = b8 ? k_bicg_spmv_alpha<T, T, 2> : k_bicg_spmv_alpha<T, T, 0>;
                EWG_LAUNCH_PDL(ctx, K_BICG_SPMV_ALPHA, kfn, G, kSolBlock, P, A, w.y, w.r0, w.v, sw->st, part, cnt, ex);
            }
            EWG_LAUNCH_PDL(ctx, K_BICG_HS, k_bicg_hs<T>, G, kSolBlock, P, w.x, w.y, w.r, w.v, sw->st, part, cnt);
            if (b8) launch_precond_b8<T>(ctx, w, relax, w.r, w.z, status);
            else launch_precond<T>(ctx, w, o->precond, relax, w.r, w.z, status);
            {
                auto kfn = b8 ? k_bicg_spmv_omega<T, T, 2> : k_bicg_spmv_omega<T, T, 0>;
                EWG_LAUNCH_PDL(ctx, K_BICG_SPMV_OMEGA, kfn, G, kSolBlock, P, A, w.z, w.r, w.y, sw->st, part, cnt, ex);
            }
            EWG_LAUNCH_PDL(ctx, K_BICG_XR, k_bicg_xr<T>, G, kSolBlock, P, w.x, w.z, w.r, w.y, w.r0, sw->st, part, cnt);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "bicgstab launch");
        if ((e = cudaMemcpyAsync(sw->h_st, sw->st, sizeof(BiState), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "read state");
        if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync bicgstab");
        if (sw->h_st->status == ST_CONVERGED && o->verify_true_residual && sw->h_st->replacements < 3) {
            auto kfn = b8 ? k_bicg_true_residual<T, T, 1> : k_bicg_true_residual<T, T, 0>;
            EWG_LAUNCH(ctx, K_BICG_TRUE_RESIDUAL, kfn, G, kSolBlock, P, A, w.b, w.x, w.r, w.r0, w.v, w.p, sw->st, part, cnt);
            if ((e = cudaMemcpyAsync(sw->h_st, sw->st, sizeof(BiState), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
                return cuda_fail(ctx, e, "read state");
            if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync true residual");
        }
        if (sw->h_st->status != ST_RUNNING) break;
        if (++guard > maxIter + 8) { ctx->err = "bicgstab: status never left RUNNING"; return EWG_ERR_TIMEOUT; }
    }
    const BiState& hs = *sw->h_st;
    *itersOut = hs.iter;
    *restartsOut = hs.restarts;
    *resOut = hs.resErr;
    *statusOut = hs.status;
    if (initOut) *initOut = hs.initResErr;
    switch (hs.status) {
        case ST_CONVERGED: return EWG_OK;
        case ST_BREAKDOWN: ctx->err = "Breakdown of the BiCGStab solver"; return EWG_ERR_BREAKDOWN;
        default: ctx->err = "BiCGStab did not converge"; return EWG_ERR_NOT_CONVERGED;
    }
}

ewg_status solver_solve(ewg_ctx* ctx, const ewg_solve_opts* o, ewg_solve_report* rep) {
    const Phys& P = ctx->P;
    const bool mixed = o->precision == EWG_PRECISION_MIXED;
    if (mixed != (ctx->jacPrecision == EWG_PRECISION_MIXED)) {
        ctx->err = "solve precision does not match the precision of the stored Jacobian";
        return EWG_ERR_INVALID;
    }
    ewg_status st = check_ordering(ctx, o);
    if (st) return st;
    st = ensure_ws(ctx, mixed);
    if (st) return st;
    SolverWs* sw = ws_of(ctx);
    const bool b8 = use_b8(ctx, o);
    cudaError_t e;
    memset(rep, 0, sizeof(*rep));
    cudaEventRecord(ctx->ev0, ctx->stream);
    int status = 0;
    if (!mixed) {
        if ((st = ensure_precond<double>(ctx, sw->d, o, EWG_PRECISION_FP64))) return st;
        if (b8) launch_b8_vector<double, double, true>(ctx, ctx->r, sw->d.b);
        else if ((e = cudaMemcpyAsync(sw->d.b, ctx->r, sizeof(double2) * P.N, cudaMemcpyDeviceToDevice, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "copy rhs");
        int it = 0, rs = 0;
        double res = 0, ini = 0;
        st = bicgstab<double>(ctx, sw->d, o, o->linear_solver_tolerance, o->linear_solver_abs_tolerance,
                              o->linear_solver_max_iterations, &it, &rs, &res, &status, &ini);
        if (st == EWG_ERR_CUDA || st == EWG_ERR_TIMEOUT) return st;
        rep->iterations = it;
        rep->restarts = rs;
        rep->outer_iterations = 1;
        rep->final_residual = res;
        rep->initial_residual = ini;
        if (b8) launch_b8_vector<double, double, false>(ctx, sw->d.x, ctx->dx);
        else if ((e = cudaMemcpyAsync(ctx->dx, sw->d.x, sizeof(double2) * P.N, cudaMemcpyDeviceToDevice, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "copy dx");
    } else {
        if ((st = ensure_precond<float>(ctx, sw->f, o, EWG_PRECISION_MIXED))) return st;
        const int G = sw->gridRed;
        int gs = grid_size_for(ctx, (const void*)k_to_float, kSolBlock);
        // x64 = 0, r64 = b
        if ((e = cudaMemsetAsync(sw->x64, 0, sizeof(double2) * P.N, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "zero x64");
        if ((e = cudaMemcpyAsync(sw->r64, ctx->r, sizeof(double2) * P.N, cudaMemcpyDeviceToDevice, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "copy r64");
        // initial max |b|
        EWG_LAUNCH(ctx, K_DEFECT_RESIDUAL, k_defect_residual, G, kSolBlock, P, ctx->J32, ctx->r, sw->x64, sw->r64, sw->partials, sw->counter, sw->dmax);
        double bmax = 0;
        if ((e = cudaMemcpyAsync(&bmax, sw->dmax, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "read bmax");
        if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync");
        rep->initial_residual = bmax;
        double init = fmax(bmax, DBL_MIN * 1e10);
        double absTol = o->defect_tolerance > 0 ? o->defect_tolerance : o->linear_solver_abs_tolerance;
        double res = bmax;
        int totalIt = 0, totalRs = 0, outer = 0;
        st = EWG_ERR_NOT_CONVERGED;
        if (res / fmax(1e-20, init) <= o->linear_solver_tolerance || res <= absTol) st = EWG_OK;
        while (st != EWG_OK && outer < o->max_defect_iterations) {
            if (b8) launch_b8_vector<double, float, true>(ctx, sw->r64, sw->f.b);
            else EWG_LAUNCH(ctx, K_TO_FLOAT, k_to_float, gs, kSolBlock, P, sw->r64, sw->f.b);
            int it = 0, rs = 0, istat = 0;
            double ires = 0;
            ewg_status ist = bicgstab<float>(ctx, sw->f, o, o->inner_tolerance, 0.0,
                                             o->linear_solver_max_iterations, &it, &rs, &ires, &istat);
            if (ist == EWG_ERR_CUDA || ist == EWG_ERR_TIMEOUT) return ist;
            totalIt += it;
            totalRs += rs;
            ++outer;
            if (ist == EWG_ERR_BREAKDOWN && it == 0) { st = EWG_ERR_BREAKDOWN; break; }
            // the inner correction back in split order (y is free after the inner solve)
            const float2* dx32 = sw->f.x;
            if (b8) {
                launch_b8_vector<float, float, false>(ctx, sw->f.x, sw->f.y);
                dx32 = sw->f.y;
            }
            EWG_LAUNCH(ctx, K_DEFECT_ACCUMULATE, k_defect_accumulate, gs, kSolBlock, P, sw->x64, dx32);
            EWG_LAUNCH(ctx, K_DEFECT_RESIDUAL, k_defect_residual, G, kSolBlock, P, ctx->J32, ctx->r, sw->x64, sw->r64, sw->partials, sw->counter, sw->dmax);
            if ((e = cudaMemcpyAsync(&res, sw->dmax, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "read defect");
            if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync defect");
            if (!(res == res)) { st = EWG_ERR_NONFINITE; ctx->err = "non-finite defect"; break; }
            if (res / fmax(1e-20, init) <= o->linear_solver_tolerance || res <= absTol) st = EWG_OK;
        }
        if (st == EWG_ERR_NOT_CONVERGED) ctx->err = "defect correction did not converge";
        rep->iterations = totalIt;
        rep->restarts = totalRs;
        rep->outer_iterations = outer;
        rep->final_residual = res;
        if ((e = cudaMemcpyAsync(ctx->dx, sw->x64, sizeof(double2) * P.N, cudaMemcpyDeviceToDevice, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "copy dx");
        status = st == EWG_OK ? ST_CONVERGED : ST_FAILED;
    }
    cudaEventRecord(ctx->ev1, ctx->stream);
    if ((e = cudaEventSynchronize(ctx->ev1)) != cudaSuccess) return cuda_fail(ctx, e, "sync solve");
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    rep->seconds = ms * 1e-3;
    rep->converged = status == ST_CONVERGED;
    rep->status = status == ST_CONVERGED ? EWG_OK : (status == ST_BREAKDOWN ? EWG_ERR_BREAKDOWN : EWG_ERR_NOT_CONVERGED);
    return (ewg_status)rep->status;
}

ewg_status solver_apply_preconditioner(ewg_ctx* ctx, const ewg_solve_opts* o, const double2* b, double2* y) {
    if (o->precision != EWG_PRECISION_FP64 || ctx->jacPrecision != EWG_PRECISION_FP64) {
        ctx->err = "apply_preconditioner is available for the FP64 Jacobian";
        return EWG_ERR_INVALID;
    }
    ewg_status st = check_ordering(ctx, o);
    if (st) return st;
    st = ensure_ws(ctx, false);
    if (st) return st;
    SolverWs* sw = ws_of(ctx);
    if ((st = ensure_precond<double>(ctx, sw->d, o, EWG_PRECISION_FP64))) return st;
    if (use_b8(ctx, o)) {
        // split-order vectors in and out: through box-8 order
        launch_b8_vector<double, double, true>(ctx, b, sw->d.t0);
        launch_precond_b8<double>(ctx, sw->d, o->preconditioner_relaxation, sw->d.t0, sw->d.t1, nullptr);
        launch_b8_vector<double, double, false>(ctx, sw->d.t1, y);
    } else {
        launch_precond<double>(ctx, sw->d, o->precond, o->preconditioner_relaxation, b, y, nullptr);
    }
    return cuda_fail(ctx, cudaGetLastError(), "apply preconditioner");
}

// One slab-iteration kernel of the distributed BiCGStab (kind: 0 p-update, 1 SpMV + dot,
// 2 h/s update, 3 SpMV + two dots, 4 x/r update); vectors in the split order, out on the device,
// st the device state (may be null for kinds 1 and 3: no status test).
ewg_status solver_slab(ewg_ctx* ctx, int kind, double2* a, double2* b, double2* c, double2* d, const double2* e,
                       const void* stv, int64_t lo, int64_t hi, double* out) {
    ewg_status st = ensure_ws(ctx, false);
    if (st) return st;
    SolverWs* sw = ws_of(ctx);
    const Phys& P = ctx->P;
    const int G = sw->gridRed;
    const BiState* bs = (const BiState*)stv;
    if (lo < 0 || hi < lo || hi > P.Nh) {
        ctx->err = "slab kernel: owned row range outside the colour half";
        return EWG_ERR_INVALID;
    }
    switch (kind) {
        case 0: EWG_LAUNCH(ctx, K_BICG_P, k_slab_p, G, kSolBlock, P, a, b, c, d, bs); break;
        case 1: EWG_LAUNCH(ctx, K_BICG_SPMV_ALPHA, k_slab_spmv_dot<0>, G, kSolBlock, P, ctx->J, a, b, c, lo, hi, bs,
                           sw->partials, sw->counter, out); break;
        case 2: EWG_LAUNCH(ctx, K_BICG_HS, k_slab_hs, G, kSolBlock, P, a, b, c, d, lo, hi, bs, sw->partials,
                           sw->counter, out); break;
        case 3: EWG_LAUNCH(ctx, K_BICG_SPMV_OMEGA, k_slab_spmv_dot2<0>, G, kSolBlock, P, ctx->J, a, b, c, lo, hi, bs,
                           sw->partials, sw->counter, out); break;
        case 4: EWG_LAUNCH(ctx, K_BICG_XR, k_slab_xr, G, kSolBlock, P, a, b, c, d, e, lo, hi, bs, sw->partials,
                           sw->counter, out); break;
        default: ctx->err = "slab kernel: unknown kind"; return EWG_ERR_INVALID;
    }
    return cuda_fail(ctx, cudaGetLastError(), "slab kernel");
}

ewg_status solver_slab_state(ewg_ctx* ctx, int stage, void* state, const double* red, const ewg_solve_opts* o) {
    if (stage < 0 || stage > 4) { ctx->err = "slab state: unknown stage"; return EWG_ERR_INVALID; }
    k_slab_state<<<1, 32, 0, ctx->stream>>>(stage, (BiState*)state, red, o ? o->linear_solver_tolerance : 0.0,
                                            o ? o->linear_solver_abs_tolerance : 0.0,
                                            o ? o->linear_solver_max_error : 0.0,
                                            o ? o->linear_solver_max_iterations : 0, o ? o->restart_on_breakdown : 0);
    return cuda_fail(ctx, cudaGetLastError(), "slab state");
}

int32_t solver_slab_state_size() { return (int32_t)sizeof(BiState); }

ewg_status solver_slab_state_read(ewg_ctx* ctx, const void* state, int32_t* status, int32_t* iterations,
                                  int32_t* restarts, double* res, double* init) {
    BiState h;
    cudaError_t e = cudaMemcpyAsync(&h, state, sizeof(BiState), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "read slab state");
    if (status) *status = h.status;
    if (iterations) *iterations = h.iter;
    if (restarts) *restarts = h.restarts;
    if (res) *res = h.resErr;
    if (init) *init = h.initResErr;
    return EWG_OK;
}

ewg_status solver_spmv(ewg_ctx* ctx, const double2* x, double2* y) {
    int g = grid_size_for(ctx, (const void*)k_spmv<double, double>, kSolBlock);
    {
        auto kfn = k_spmv<double, double>;
        EWG_LAUNCH(ctx, K_SPMV, kfn, g, kSolBlock, ctx->P, ctx->J, x, y);
    }
    return cuda_fail(ctx, cudaGetLastError(), "spmv");
}

ewg_status solver_newton_update(ewg_ctx* ctx, int* nonfinite) {
    ewg_status st = ensure_ws(ctx, false);
    if (st) return st;
    SolverWs* sw = ws_of(ctx);
    cudaError_t e;
    if ((e = cudaMemsetAsync(sw->flags + 1, 0, sizeof(int), ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "memset");
    int g = grid_size_for(ctx, (const void*)k_newton_update, kSolBlock);
    EWG_LAUNCH(ctx, K_NEWTON_UPDATE, k_newton_update, g, kSolBlock, ctx->P, ctx->x0, ctx->dx, sw->flags + 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "newton update");
    int bad = 0;
    if ((e = cudaMemcpyAsync(&bad, sw->flags + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "read");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync update");
    *nonfinite = bad;
    return EWG_OK;
}

}  // namespace ewg
