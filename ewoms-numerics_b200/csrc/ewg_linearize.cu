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

// One interior face seen from the focus cell i (darcyfluxmodule.hh:185-324, 461-527;
// immisciblelocalresidual.hh:123-149): adds the mass fluxes to R_i and dR_i/dx_i and returns the
// block dR_j/dx_i of the neighbour's local residual (already divided by the neighbour's volume).
template <int AXIS>
__device__ __forceinline__ void interior_face(const Phys& P, int side, int idxA, double Ki, const double pI[2],
                                              double dpcI, const double lam[2], const double dlam[2],
                                              double2 xj, double Kj, double pcj, const double lamj[2],
                                              double R[2], double D[2][2], double Dj[4]) {
    const double h = P.h[AXIS];
    const double xc = (idxA + 0.5) * h;
    const double xcj = (idxA + (side ? 1 : -1) + 0.5) * h;
    const double dA = xcj - xc;
    const double distSq = dA * dA;
    const double coef = dA / distSq;
    const double nA = side ? 1.0 : -1.0;
    const double Kf = harmonic_mean(Ki, Kj);
    const double area = P.area[AXIS];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const double pJ = a == 0 ? xj.x : xj.x + (pcj - 0.0);
        const double deltay = pJ - pI[a];
        double grad = deltay * coef;
        const double dgP = -coef;
        const double dgS = a == 0 ? 0.0 : -dpcI * coef;
        if (AXIS == 1) {
            // gravity correction; for the other axes the hydrostatic terms are exactly zero
            const double xf = (idxA + side) * h;
            const double gIn = -P.g * (xc - xf), gEx = -P.g * (xcj - xf);
            const double rho = P.rho[a];
            const double pStatIn = -rho * gIn;
            const double pStatEx = -(rho * gEx);
            grad = grad + dA * ((pStatEx - pStatIn) / distSq);
        }
        const bool upExt = grad * nA > 0;
        const double lamU = upExt ? lamj[a] : lam[a];
        const double dlamU = upExt ? 0.0 : dlam[a];
        const double sK = Kf * grad;
        const double vel = sK * (-lamU);
        const double dvelP = (Kf * dgP) * (-lamU);
        const double dvelS = (Kf * dgS) * (-lamU) + (-dlamU) * sK;
        const double rho = P.rho[a];
        const double F = vel * nA * rho * area;
        const double dFP = dvelP * nA * rho * area;
        const double dFS = dvelS * nA * rho * area;
        R[a] += F;
        D[a][0] += dFP;
        D[a][1] += dFS;
        Dj[2 * a] = -dFP / P.vol;
        Dj[2 * a + 1] = -dFS / P.vol;
    }
}

// One boundary face of the lens problem (lensproblem.hh:464-533): free flow with the hydrostatic
// S_w = 1 state on the left / right faces (immiscibleboundaryratevector.hh:91-153, boundary
// gradient fvbasegradientcalculator.hh:277-312, darcyfluxmodule.hh:333-453), the DNAPL inlet on
// the top face, no flow elsewhere.
template <int DIM, int AXIS>
__device__ __forceinline__ void boundary_face(const Phys& P, int side, const int idx[3], int lensI, double Ki,
                                              const double pI[2], double dpcI, const double lam[2],
                                              const double dlam[2], double R[2], double D[2][2]) {
    double xc[3], xf[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) xc[d] = d < DIM ? (idx[d] + 0.5) * P.h[d] : 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) xf[d] = xc[d];
    xf[AXIS] = (idx[AXIS] + side) * P.h[AXIS];
    const double area = P.area[AXIS];
    const bool left = xf[0] < 0.0 + P.eps, right = xf[0] > P.L[0] - P.eps;
    if (left || right) {
        const double g1 = -P.g;
        const double depth = P.L[1] - xf[1];
        const double pw = left ? P.pRef - P.leftScale * P.rho[0] * g1 * depth : P.pRef - P.rho[0] * g1 * depth;
        const double pB[2] = {pw, pw + P.bndPc[in_lens(P, xf) ? 1 : 0] - 0.0};
        const double dA = xf[AXIS] - xc[AXIS];
        const double distSq = dA * dA;
        const double distIn = xc[AXIS] - xf[AXIS];
        const double absDistSq = distIn * distIn;
        const double gTimesDist = AXIS == 1 ? g1 * distIn : 0.0;
        const double coef = dA / distSq;
        const double nA = side ? 1.0 : -1.0;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const double deltay = pB[a] - pI[a];
            double grad = deltay * coef;
            const double dgP = -coef;
            const double dgS = a == 0 ? 0.0 : -dpcI * coef;
            const double rho = P.rho[a];
            const double pStatIn = -gTimesDist * rho;
            grad = grad + distIn * (pStatIn / absDistSq);
            const bool upB = grad * nA > 0;
            const double lamU = upB ? P.bndLam[lensI][a] : lam[a];
            const double dlamU = upB ? 0.0 : dlam[a];
            const double sK = Ki * grad;
            const double vel = sK * (-lamU);
            const double dvelP = (Ki * dgP) * (-lamU);
            const double dvelS = (Ki * dgS) * (-lamU) + (-dlamU) * sK;
            R[a] += vel * nA * rho * area;
            D[a][0] += dvelP * nA * rho * area;
            D[a][1] += dvelS * nA * rho * area;
        }
        return;
    }
    const bool upper = xf[1] > P.L[1] - P.eps;
    bool inlet = upper && xf[0] > P.inletXlo && xf[0] < P.inletXhi;
    if (DIM == 3) inlet = inlet && xf[2] > P.inletZlo && xf[2] < P.inletZhi;
    if (inlet) R[1] += P.inletRate * area;
}

template <int DIM, typename JT, bool WITH_J>
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
        const int nAx[3] = {P.nx, P.ny, P.nz};
        const double2 xi = x[s];
        const double Ki = perm[s];
        const double pci = iq[s], dpci = iq[N + s];
        const double lam[2] = {iq[2 * N + s], iq[4 * N + s]};
        const double dlam[2] = {iq[3 * N + s], iq[5 * N + s]};
        // p_alpha = p_w + (pC[alpha] - pC[0]) with pC[0] = 0
        const double pI[2] = {xi.x, xi.x + (pci - 0.0)};

        double R[2] = {0.0, 0.0};
        double D[2][2] = {{0.0, 0.0}, {0.0, 0.0}};

        const bool interior = ci.i > 0 && ci.i < P.nx - 1 && ci.j > 0 && ci.j < P.ny - 1 &&
                              (DIM == 2 || (ci.k > 0 && ci.k < P.nz - 1));
        if (interior) {
            // every face has a neighbour: issue all neighbour loads before the flux arithmetic
            constexpr int NF = 2 * DIM;
            const int64_t base = (int64_t)(col ^ 1) * P.Nh;
            int64_t nb[NF];
            nb[0] = base + h - 1 + ci.b;
            nb[1] = base + h + ci.b;
            nb[2] = base + h - P.nxh;
            nb[3] = base + h + P.nxh;
            if (DIM == 3) {
                nb[NF - 2] = base + h - P.planeh;
                nb[NF - 1] = base + h + P.planeh;
            }
            const double* xs = reinterpret_cast<const double*>(x);
            double pwj[NF], Kj[NF], pcj[NF], lwj[NF], lnj[NF];
#pragma unroll
            for (int q = 0; q < NF; ++q) {
                pwj[q] = xs[2 * nb[q]];
                Kj[q] = perm[nb[q]];
                pcj[q] = iq[nb[q]];
                lwj[q] = iq[2 * N + nb[q]];
                lnj[q] = iq[4 * N + nb[q]];
            }
#pragma unroll
            for (int q = 0; q < NF; ++q) {
                const int axis = q >> 1, side = q & 1;
                const double lamj[2] = {lwj[q], lnj[q]};
                const double2 xj = make_double2(pwj[q], 0.0);
                double Dj[4];
                if (axis == 0)
                    interior_face<0>(P, side, idx[0], Ki, pI, dpci, lam, dlam, xj, Kj[q], pcj[q], lamj, R, D, Dj);
                else if (axis == 1)
                    interior_face<1>(P, side, idx[1], Ki, pI, dpci, lam, dlam, xj, Kj[q], pcj[q], lamj, R, D, Dj);
                else
                    interior_face<2>(P, side, idx[2], Ki, pI, dpci, lam, dlam, xj, Kj[q], pcj[q], lamj, R, D, Dj);
                if (WITH_J) store_block(J, N, opposite_band(band_of(axis, side)), nb[q], Dj);
            }
        } else {
        // ---- fluxes over interior faces in intersection order (-x, +x, -y, +y, -z, +z) ----
#pragma unroll
        for (int axis = 0; axis < DIM; ++axis) {
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int64_t sj = neighbour_split(P, col, h, ci, axis, side);
                if (sj < 0) continue;
                const double2 xj = x[sj];
                const double Kj = perm[sj];
                const double pcj = iq[sj];
                const double lamj[2] = {iq[2 * N + sj], iq[4 * N + sj]};
                double Dj[4];
                if (axis == 0)
                    interior_face<0>(P, side, idx[0], Ki, pI, dpci, lam, dlam, xj, Kj, pcj, lamj, R, D, Dj);
                else if (axis == 1)
                    interior_face<1>(P, side, idx[1], Ki, pI, dpci, lam, dlam, xj, Kj, pcj, lamj, R, D, Dj);
                else
                    interior_face<2>(P, side, idx[2], Ki, pI, dpci, lam, dlam, xj, Kj, pcj, lamj, R, D, Dj);
                if (WITH_J) store_block(J, N, opposite_band(band_of(axis, side)), sj, Dj);
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
        if (!interior)
#pragma unroll
        for (int axis = 0; axis < DIM; ++axis) {
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const bool has = side == 0 ? idx[axis] > 0 : idx[axis] < nAx[axis] - 1;
                if (has) continue;
                const int li = lens[s];
                if (axis == 0)
                    boundary_face<DIM, 0>(P, side, idx, li, Ki, pI, dpci, lam, dlam, R, D);
                else if (axis == 1)
                    boundary_face<DIM, 1>(P, side, idx, li, Ki, pI, dpci, lam, dlam, R, D);
                else
                    boundary_face<DIM, 2>(P, side, idx, li, Ki, pI, dpci, lam, dlam, R, D);
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

// S_w = 1 state of the free-flow boundary per region: p_cnw and k_r / mu of both phases
__global__ void k_boundary_constants(const __grid_constant__ Phys P, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int r = 0; r < 2; ++r) {
        MatOut m = material(P.law[r], 1.0);
        out[3 * r] = m.pc.v;
        out[3 * r + 1] = m.krw.v / P.mu[0];
        out[3 * r + 2] = m.krn.v / P.mu[1];
    }
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

ewg_status compute_boundary_constants(ewg_ctx* ctx) {
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * 6);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "alloc boundary constants");
    k_boundary_constants<<<1, 32, 0, ctx->stream>>>(ctx->P, d);
    double h[6] = {0, 0, 0, 0, 0, 0};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "boundary constants");
    for (int r = 0; r < 2; ++r) {
        ctx->P.bndPc[r] = h[3 * r];
        ctx->P.bndLam[r][0] = h[3 * r + 1];
        ctx->P.bndLam[r][1] = h[3 * r + 2];
    }
    return EWG_OK;
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
    const bool three = ctx->P.dim == 3;
    if (!withJacobian) {
        auto k = three ? k_assemble<3, double, false> : k_assemble<2, double, false>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                                             nullptr, ctx->d_errmax, ctx->d_flags);
    } else if (ctx->jacPrecision == EWG_PRECISION_MIXED) {
        auto k = three ? k_assemble<3, float, true> : k_assemble<2, float, true>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                                             ctx->J32, ctx->d_errmax, ctx->d_flags);
    } else {
        auto k = three ? k_assemble<3, double, true> : k_assemble<2, double, true>;
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
