// ECFV + AD linearization of the immiscible two-phase model on the device.
//
// Replaces FvBaseLinearizer::linearize_ / linearizeElement_ (fvbaselinearizer.hh:401-512) with
// FvBaseAdLocalLinearizer (fvbaseadlocallinearizer.hh:178-297). As in the reference's ECFV path,
// the element of cell i focuses on its own DOF, evaluates its local residual with derivatives with
// respect to x_i only, writes its residual row r_i and scatters the Jacobian *column* i:
// J[i][i] and J[j][i] for every face neighbour j. Column ownership makes the scatter atomic-free
// without colouring (the reference needs no lock for ECFV either, ecfvdiscretization.hh:109): one
// thread owns one cell, and the blocks J[j][i] it writes are written by nobody else.
//
// Two kernels per linearization:
//   k_intensive  one thread per cell: the intensive quantities of immiscibleintensivequantities.hh
//                :87-145 that neighbours need (p_c, lambda_w, lambda_n with d/dS_w), written once
//                per cell like the reference's intensive-quantity cache (lensproblem.hh:166).
//   k_assemble   one thread per cell: fluxes over its faces (darcyfluxmodule.hh:185-527,
//                immisciblelocalresidual.hh:123-149), the implicit-Euler storage term
//                (fvbaselocalresidual.hh:494-629), the lens boundary conditions
//                (lensproblem.hh:464-533, immiscibleboundaryratevector.hh:91-153), division by
//                the cell volume, and the residual max-norm of NewtonMethod::preSolve_.
#include <cstdio>

#include "ewg_physics.cuh"

namespace ewg {

constexpr int kLinBlock = 256;

__global__ void __launch_bounds__(kLinBlock) k_intensive(const __grid_constant__ Phys P,
                                                         const double2* __restrict__ x,
                                                         const uint8_t* __restrict__ lens,
                                                         double* __restrict__ iq) {
    const int64_t N = P.N;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const double Sw = x[s].y;
        const LawDev& L = P.law[lens[s]];
        MatOut m = material(L, Sw);
        // mobility = kr / mu as an AD quotient with a constant denominator
        double muw = P.mu[0], mun = P.mu[1];
        iq[s] = m.pc.v;
        iq[N + s] = m.pc.d;
        iq[2 * N + s] = m.krw.v / muw;
        iq[3 * N + s] = (muw * m.krw.d) / (muw * muw);
        iq[4 * N + s] = m.krn.v / mun;
        iq[5 * N + s] = (mun * m.krn.d) / (mun * mun);
    }
}

__device__ __forceinline__ void store_block(double* J, int64_t N, int band, int64_t s, const double b[4]) {
    double* base = J + (int64_t)band * 4 * N + s;
    base[0] = b[0];
    base[N] = b[1];
    base[2 * N] = b[2];
    base[3 * N] = b[3];
}
__device__ __forceinline__ void store_block(float* J, int64_t N, int band, int64_t s, const double b[4]) {
    float* base = J + (int64_t)band * 4 * N + s;
    base[0] = (float)b[0];
    base[N] = (float)b[1];
    base[2 * N] = (float)b[2];
    base[3 * N] = (float)b[3];
}

// Non-negative doubles compare like their bit patterns as unsigned integers.
__device__ __forceinline__ void block_max_publish(double v, unsigned long long* out) {
    __shared__ double sm[kLinBlock / 32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? sm[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

template <typename JT, bool WITH_J>
__global__ void __launch_bounds__(kLinBlock) k_assemble(
    const __grid_constant__ Phys P, const double2* __restrict__ x, const double2* __restrict__ sold,
    const double* __restrict__ perm, const uint8_t* __restrict__ lens, const double* __restrict__ iq,
    double dt, double2* __restrict__ rOut, JT* __restrict__ J, unsigned long long* errmax,
    int* flags) {
    const int64_t N = P.N;
    const double V = P.vol;
    double localMax = 0.0;
    int bad = 0;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int col = s >= P.Nh ? 1 : 0;
        const int64_t h = s - col * P.Nh;
        const CellIdx ci = cell_of(P, col, h);
        const int idx[3] = {ci.i, ci.j, ci.k};
        const double2 xi = x[s];
        const double Ki = perm[s];
        const double pci = iq[s], dpci = iq[N + s];
        const double lam[2] = {iq[2 * N + s], iq[4 * N + s]};
        const double dlam[2] = {iq[3 * N + s], iq[5 * N + s]};
        // p_alpha = p_w + (pC[alpha] - pC[0]) with pC[0] = 0
        const double pI[2] = {xi.x + (0.0 - 0.0), xi.x + (pci - 0.0)};
        const double dpIdS[2] = {0.0, dpci};
        double xc[3];
        for (int a = 0; a < 3; ++a) xc[a] = a < P.dim ? (idx[a] + 0.5) * P.h[a] : 0.0;
        const double g[3] = {0.0, -P.g, 0.0};

        // residual of the focus DOF and its derivatives [eq][pv]
        double R[2] = {0.0, 0.0};
        double D[2][2] = {{0.0, 0.0}, {0.0, 0.0}};

        // ---- fluxes over interior faces (YaspGrid intersection order) ----
        for (int axis = 0; axis < P.dim; ++axis) {
            for (int side = 0; side < 2; ++side) {
                const int64_t sj = neighbour_split(P, col, h, ci, axis, side);
                if (sj < 0) continue;
                const double2 xj = x[sj];
                const double Kj = perm[sj];
                const double pcj = iq[sj];
                const double lamj[2] = {iq[2 * N + sj], iq[4 * N + sj]};
                double xcj[3] = {xc[0], xc[1], xc[2]};
                xcj[axis] = (idx[axis] + (side ? 1 : -1) + 0.5) * P.h[axis];
                double xf[3] = {xc[0], xc[1], xc[2]};
                xf[axis] = (idx[axis] + side) * P.h[axis];
                double distSq = 0.0, gIn = 0.0, gEx = 0.0;
                for (int d = 0; d < P.dim; ++d) {
                    double t = xcj[d] - xc[d];
                    distSq += t * t;
                }
                for (int d = 0; d < P.dim; ++d) {
                    gIn += g[d] * (xc[d] - xf[d]);
                    gEx += g[d] * (xcj[d] - xf[d]);
                }
                const double dA = xcj[axis] - xc[axis];
                const double coef = dA / distSq;
                const double nA = side ? 1.0 : -1.0;
                const double Kf = harmonic_mean(Ki, Kj);
                const double area = P.area[axis];
                double Dj[2][2];
                for (int a = 0; a < 2; ++a) {
                    const double pJ = a == 0 ? xj.x + (0.0 - 0.0) : xj.x + (pcj - 0.0);
                    // raw two-point gradient along the face axis, derivatives from the focus only
                    const double deltay = pJ - pI[a];
                    double grad = deltay * coef;
                    const double dgP = -1.0 * coef;
                    const double dgS = -dpIdS[a] * coef;
                    // gravity correction with the phase densities of both sides
                    const double rho = P.rho[a];
                    const double pStatIn = -rho * gIn;
                    const double pStatEx = -(rho * gEx);
                    grad = grad + dA * ((pStatEx - pStatIn) / distSq);
                    const double tmp = grad * nA;
                    const bool upExt = tmp > 0;
                    const double lamU = upExt ? lamj[a] : lam[a];
                    const double dlamU = upExt ? 0.0 : dlam[a];
                    // filter velocity -lambda K grad, volume flux v.n, mass flux * rho_up * area
                    const double sK = Kf * grad;
                    const double vel = sK * (-lamU);
                    const double dvelP = (Kf * dgP) * (-lamU);
                    const double dvelS = (Kf * dgS) * (-lamU) + (-dlamU) * sK;
                    const double F = vel * nA * rho * area;
                    const double dFP = dvelP * nA * rho * area;
                    const double dFS = dvelS * nA * rho * area;
                    R[a] += F;
                    D[a][0] += dFP;
                    D[a][1] += dFS;
                    Dj[a][0] = -dFP / V;
                    Dj[a][1] = -dFS / V;
                }
                if (WITH_J) {
                    const double blk[4] = {Dj[0][0], Dj[0][1], Dj[1][0], Dj[1][1]};
                    store_block(J, N, opposite_band(band_of(axis, side)), sj, blk);
                }
            }
        }

        // ---- storage: (phi S rho - storage(x_old)) V / dt ----
        {
            const double2 so = sold[s];
            const double Sw = xi.y;
            const double fac = V / dt;
            const double sw0 = P.porosity * Sw * P.rho[0];
            const double sn0 = P.porosity * (1.0 - (0.0 + Sw)) * P.rho[1];
            R[0] += (sw0 - so.x) * fac;
            R[1] += (sn0 - so.y) * fac;
            D[0][1] += (P.porosity * P.rho[0]) * fac;
            D[1][1] += (-P.porosity * P.rho[1]) * fac;
        }

        // ---- boundary faces ----
        for (int axis = 0; axis < P.dim; ++axis) {
            for (int side = 0; side < 2; ++side) {
                const bool has = side == 0 ? idx[axis] > 0 : idx[axis] < (axis == 0 ? P.nx : (axis == 1 ? P.ny : P.nz)) - 1;
                if (has) continue;
                double xf[3] = {xc[0], xc[1], xc[2]};
                xf[axis] = (idx[axis] + side) * P.h[axis];
                const double area = P.area[axis];
                const bool left = xf[0] < 0.0 + P.eps, right = xf[0] > P.L[0] - P.eps;
                if (left || right) {
                    // free-flow boundary with a hydrostatic fluid state at S_w = 1
                    const double depth = P.L[1] - xf[1];
                    const double pw = left ? P.pRef - P.leftScale * P.rho[0] * g[1] * depth
                                           : P.pRef - P.rho[0] * g[1] * depth;
                    const MatOut mf = material(P.law[in_lens(P, xf) ? 1 : 0], 1.0);
                    const MatOut mi = material(P.law[lens[s]], 1.0);
                    const double pB[2] = {pw, pw + mf.pc.v - 0.0};
                    const double lamB[2] = {mi.krw.v / P.mu[0], mi.krn.v / P.mu[1]};
                    double distSq = 0.0, absDistSq = 0.0, gTimesDist = 0.0;
                    for (int d = 0; d < P.dim; ++d) {
                        double t = xf[d] - xc[d];
                        distSq += t * t;
                        double u = xc[d] - xf[d];
                        absDistSq += u * u;
                        gTimesDist += g[d] * u;
                    }
                    const double coef = (xf[axis] - xc[axis]) / distSq;
                    const double distIn = xc[axis] - xf[axis];
                    const double nA = side ? 1.0 : -1.0;
                    for (int a = 0; a < 2; ++a) {
                        const double deltay = pB[a] - pI[a];
                        double grad = deltay * coef;
                        const double dgP = -1.0 * coef;
                        const double dgS = -dpIdS[a] * coef;
                        const double rho = P.rho[a];
                        const double pStatIn = -gTimesDist * rho;
                        grad = grad + distIn * (pStatIn / absDistSq);
                        const double tmp = grad * nA;
                        const bool upB = tmp > 0;
                        const double lamU = upB ? lamB[a] : lam[a];
                        const double dlamU = upB ? 0.0 : dlam[a];
                        const double sK = Ki * grad;
                        const double vel = sK * (-lamU);
                        const double dvelP = (Ki * dgP) * (-lamU);
                        const double dvelS = (Ki * dgS) * (-lamU) + (-dlamU) * sK;
                        R[a] += vel * nA * rho * area;
                        D[a][0] += dvelP * nA * rho * area;
                        D[a][1] += dvelS * nA * rho * area;
                    }
                    continue;
                }
                const bool upper = xf[1] > P.L[1] - P.eps;
                bool inlet = upper && xf[0] > P.inletXlo && xf[0] < P.inletXhi;
                if (inlet && P.dim == 3) inlet = xf[2] > P.inletZlo && xf[2] < P.inletZhi;
                if (inlet) R[1] += P.inletRate * area;
            }
        }

        // ---- volumetric residual and stores ----
        R[0] /= V;
        R[1] /= V;
        rOut[s] = make_double2(R[0], R[1]);
        if (WITH_J) {
            const double blk[4] = {D[0][0] / V, D[0][1] / V, D[1][0] / V, D[1][1] / V};
            store_block(J, N, 0, s, blk);
        }
        const double e = fmax(fabs(R[0]), fabs(R[1]));
        if (!(fabs(R[0]) <= 1.7976931348623157e308) || !(fabs(R[1]) <= 1.7976931348623157e308)) bad = 1;
        localMax = fmax(localMax, e);
    }
    if (bad) atomicOr(flags, 1);
    block_max_publish(localMax, errmax);
}

__global__ void k_storage(const __grid_constant__ Phys P, const double2* __restrict__ x,
                          double2* __restrict__ sold) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const double Sw = x[s].y;
        sold[s] = make_double2(P.porosity * Sw * P.rho[0], P.porosity * (1.0 - (0.0 + Sw)) * P.rho[1]);
    }
}

// LensProblem::initial: hydrostatic p_w = p_ref - rho_w g_y depth, S_w = 1
__global__ void k_initial(const __grid_constant__ Phys P, double2* __restrict__ x) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int col = s >= P.Nh ? 1 : 0;
        const CellIdx ci = cell_of(P, col, s - col * P.Nh);
        const double y = (ci.j + 0.5) * P.h[1];
        const double depth = P.L[1] - y;
        const double densityW = P.rho[0];
        x[s] = make_double2(P.pRef - densityW * (-P.g) * depth, 1.0);
    }
}

ewg_status launch_storage(ewg_ctx* ctx, const double2* x, double2* sold) {
    int grid = grid_size_for(ctx, (const void*)k_storage, kLinBlock);
    EWG_LAUNCH(ctx, K_STORAGE, k_storage, grid, kLinBlock, ctx->P, x, sold);
    return cuda_fail(ctx, cudaGetLastError(), "k_storage");
}

ewg_status launch_initial_solution(ewg_ctx* ctx, double2* x) {
    int grid = grid_size_for(ctx, (const void*)k_initial, kLinBlock);
    EWG_LAUNCH(ctx, K_INITIAL, k_initial, grid, kLinBlock, ctx->P, x);
    return cuda_fail(ctx, cudaGetLastError(), "k_initial");
}

ewg_status launch_linearize(ewg_ctx* ctx, double dt, bool withJacobian, const double2* x,
                            double2* r, double* maxOut, int* nonfinite) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(ctx->d_errmax, 0, sizeof(unsigned long long), ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "memset errmax");
    if ((e = cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "memset flags");
    int g1 = grid_size_for(ctx, (const void*)k_intensive, kLinBlock);
    EWG_LAUNCH(ctx, K_INTENSIVE, k_intensive, g1, kLinBlock, ctx->P, x, ctx->lens, ctx->iq);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "k_intensive");
    if (!withJacobian) {
        auto k = k_assemble<double, false>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                                             nullptr, ctx->d_errmax, ctx->d_flags);
    } else if (ctx->jacPrecision == EWG_PRECISION_MIXED) {
        auto k = k_assemble<float, true>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                                             ctx->J32, ctx->d_errmax, ctx->d_flags);
    } else {
        auto k = k_assemble<double, true>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                                             ctx->J, ctx->d_errmax, ctx->d_flags);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "k_assemble");
    if (maxOut || nonfinite) {
        // small synchronous read-back: the Newton loop needs the error on the host
        unsigned long long bits = 0;
        int flag = 0;
        if ((e = cudaMemcpyAsync(&bits, ctx->d_errmax, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "read errmax");
        if ((e = cudaMemcpyAsync(&flag, ctx->d_flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
            return cuda_fail(ctx, e, "read flags");
        if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(ctx, e, "sync linearize");
        double v;
        memcpy(&v, &bits, sizeof(v));
        if (maxOut) *maxOut = v;
        if (nonfinite) *nonfinite = flag;
    }
    return EWG_OK;
}

}  // namespace ewg
