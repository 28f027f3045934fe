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
//                :87-145 that neighbours need (p_c, lambda_w, lambda_n; on 2D grids also their
//                d/dS_w), written once per cell like the reference's intensive-quantity cache
//                (lensproblem.hh:166). The 3D assembly evaluates its own cell's quantities with
//                their derivatives itself; cells at S_w = 1 take them from a per-region table.
//   k_assemble   one thread per cell: fluxes over its faces (darcyfluxmodule.hh:185-527,
//                immisciblelocalresidual.hh:123-149), the implicit-Euler storage term
//                (fvbaselocalresidual.hh:494-629), the lens boundary conditions
//                (lensproblem.hh:464-533, immiscibleboundaryratevector.hh:91-153), division by
//                the cell volume, and the residual max-norm of NewtonMethod::preSolve_.
#include <cstdio>
#include <vector>

#include "ewg_assemble.cuh"

namespace ewg {

constexpr int kLinBlock = 256;

__global__ void __launch_bounds__(kLinBlock) k_intensive(const __grid_constant__ Phys P,
                                                         const double2* __restrict__ x,
                                                         const uint8_t* __restrict__ lens,
                                                         double* __restrict__ iq) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x)
        intensive_cell(P, x, lens, iq, s, P.dim == 2);  // 3D kernels evaluate their own cell
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

// General per-cell kernel (2D grids): runtime face loops, geometry from cell positions.
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


// 3D grids: every cell through assemble_cell3 (face geometry from the table)
// threads per block of the 3D assembly (with EWG_INTERIOR_MIN_BLOCKS below: 256 threads, two
// blocks per SM, 99 registers without spills measured fastest against 128 x 4-5 and 192 x 3)
#ifndef EWG_ASSEMBLE3_BLOCK
#define EWG_ASSEMBLE3_BLOCK 256
#endif
constexpr int kAsm3Block = EWG_ASSEMBLE3_BLOCK;

template <typename JT, bool WITH_J, int MINB>
__global__ void __launch_bounds__(kAsm3Block, MINB) k_assemble3(
    const __grid_constant__ Phys P, const FaceGeo* __restrict__ geo, const double2* __restrict__ x,
    const double2* __restrict__ sold, const double* __restrict__ perm, const uint8_t* __restrict__ lens,
    const double* __restrict__ iq, double dt, double2* __restrict__ rOut, JT* __restrict__ J,
    unsigned long long* errmax, int* flags) {
    double localMax = 0.0;
    int bad = 0;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N;
         s += (int64_t)gridDim.x * blockDim.x)
        localMax = fmax(localMax, assemble_cell3<JT, WITH_J>(P, geo, x, sold, perm, lens, iq, dt, rOut, J, s, bad,
                                                             nbr_global(x, perm, iq, P.N)));
    if (bad) atomicOr(flags, 1);
    block_max_publish(localMax, errmax);
}

// ---- finite-difference local linearizer ---------------------------------------------------------
//
// FvBaseFdLocalLinearizer (fvbasefdlocallinearizer.hh:221-237, 393-453): the local residual of
// the element of cell i (its own row and the face-flux contributions to its neighbours' rows) is
// evaluated at the primary variables and at the own primary variable deflected by
// eps = BaseEpsilon / primaryVarWeight (0.9123e-10; weight 10 / p_ref for the pressure, 1 for the
// saturation, immisciblemodel.hh:298-310), and the Jacobian column i is the difference quotient
// (NumericDifferenceMethod +1 forward, 0 central, -1 backward). Values only: the deflected own
// intensive quantities are re-evaluated, the neighbours' come from the cache.

struct FdState {
    double pw, Sw, pc, lw, ln;
};

// local residual of element s at own state st: own row R (volumetric) and the neighbour rows Fn
// per face slot (band order -x, +x, -y, +y[, -z, +z]; zero where no neighbour)
template <int DIM>
__device__ __forceinline__ void fd_local_residual(const Phys& P, int col, int64_t h, const CellIdx& ci,
                                                  const FdState& st, double Ki, int lensI, double2 so, double dt,
                                                  const double2* __restrict__ x, const double* __restrict__ perm,
                                                  const double* __restrict__ iq, double R[2], double Fn[6][2]) {
    const int64_t N = P.N;
    const int idx[3] = {ci.i, ci.j, ci.k};
    const double pI[2] = {st.pw, st.pw + (st.pc - 0.0)};
    const double lam[2] = {st.lw, st.ln};
    const double zero2[2] = {0.0, 0.0};
    double Ddummy[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    R[0] = R[1] = 0.0;
#pragma unroll
    for (int axis = 0; axis < DIM; ++axis) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const int q = 2 * axis + side;
            Fn[q][0] = Fn[q][1] = 0.0;
            const int64_t sj = neighbour_split(P, col, h, ci, axis, side);
            if (sj < 0) continue;
            const double2 xj = x[sj];
            const double lamj[2] = {iq[2 * N + sj], iq[4 * N + sj]};
            double F[2] = {0.0, 0.0};
            double Dj[4];
            if (axis == 0)
                interior_face<0>(P, side, idx[0], Ki, pI, 0.0, lam, zero2, xj, perm[sj], iq[sj], lamj, F, Ddummy, Dj);
            else if (axis == 1)
                interior_face<1>(P, side, idx[1], Ki, pI, 0.0, lam, zero2, xj, perm[sj], iq[sj], lamj, F, Ddummy, Dj);
            else
                interior_face<2>(P, side, idx[2], Ki, pI, 0.0, lam, zero2, xj, perm[sj], iq[sj], lamj, F, Ddummy, Dj);
            R[0] += F[0];
            R[1] += F[1];
            Fn[q][0] = (0.0 - F[0]) / P.vol;
            Fn[q][1] = (0.0 - F[1]) / P.vol;
        }
    }
    {
        const double fac = P.vol / dt;
        const double sw0 = P.porosity * st.Sw * P.rho[0];
        const double sn0 = P.porosity * (1.0 - (0.0 + st.Sw)) * P.rho[1];
        R[0] += (sw0 - so.x) * fac;
        R[1] += (sn0 - so.y) * fac;
    }
    const int nAx[3] = {P.nx, P.ny, P.nz};
#pragma unroll
    for (int axis = 0; axis < DIM; ++axis) {
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const bool has = side == 0 ? idx[axis] > 0 : idx[axis] < nAx[axis] - 1;
            if (has) continue;
            if (axis == 0)
                boundary_face<DIM, 0>(P, side, idx, lensI, Ki, pI, 0.0, lam, zero2, R, Ddummy);
            else if (axis == 1)
                boundary_face<DIM, 1>(P, side, idx, lensI, Ki, pI, 0.0, lam, zero2, R, Ddummy);
            else
                boundary_face<DIM, 2>(P, side, idx, lensI, Ki, pI, 0.0, lam, zero2, R, Ddummy);
        }
    }
    R[0] /= P.vol;
    R[1] /= P.vol;
}

// (a pressure deflection keeps the intensive quantities of the primary variables, which the
// callers take from the cache: the same values)
template <int DIM>
__device__ __forceinline__ FdState fd_state(const Phys& P, const LawDev& L, double pw, double Sw) {
    const MatOut m = material(L, Sw);
    return FdState{pw, Sw, m.pc.v, m.krw.v / P.mu[0], m.krn.v / P.mu[1]};
}

template <int DIM, typename JT>
__global__ void __launch_bounds__(kLinBlock) k_assemble_fd(
    const __grid_constant__ Phys P, const double2* __restrict__ x, const double2* __restrict__ sold,
    const double* __restrict__ perm, const uint8_t* __restrict__ lens, const double* __restrict__ iq, double dt,
    double refPressure, int method, double2* __restrict__ rOut, JT* __restrict__ J, unsigned long long* errmax,
    int* flags) {
    const int64_t N = P.N;
    const double baseEps = fmax(0.9123e-10, 2.220446049250313e-16 * 1.23e3);
    double localMax = 0.0;
    int bad = 0;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < N;
         s += (int64_t)gridDim.x * blockDim.x) {
        const int col = s >= P.Nh ? 1 : 0;
        const int64_t h = s - col * P.Nh;
        const CellIdx ci = cell_of(P, col, h);
        const double2 xi = x[s];
        const double Ki = perm[s];
        const int li = lens[s];
        const double2 so = sold[s];
        const FdState base{xi.x, xi.y, iq[s], iq[2 * N + s], iq[4 * N + s]};
        double R0[2], F0[6][2];
        fd_local_residual<DIM>(P, col, h, ci, base, Ki, li, so, dt, x, perm, iq, R0, F0);
        rOut[s] = make_double2(R0[0], R0[1]);
        const double e = fmax(fabs(R0[0]), fabs(R0[1]));
        if (!(fabs(R0[0]) <= 1.7976931348623157e308) || !(fabs(R0[1]) <= 1.7976931348623157e308)) bad = 1;
        localMax = fmax(localMax, e);
        double Jd[4];
        double Jn[6][4];
#pragma unroll
        for (int pv = 0; pv < 2; ++pv) {
            const double pvWeight = pv == 0 ? 10 / refPressure : 1.0;
            const double eps = baseEps / pvWeight;
            double pri[2] = {xi.x, xi.y};
            double delta = 0.0;
            double dR[2], dF[6][2];
            double Rp[2], Fp[6][2];
            if (method >= 0) {
                pri[pv] += eps;
                delta += eps;
                fd_local_residual<DIM>(P, col, h, ci, (pv == 0 ? FdState{pri[0], pri[1], base.pc, base.lw, base.ln} : fd_state<DIM>(P, P.law[li], pri[0], pri[1])), Ki, li, so, dt, x,
                                       perm, iq, Rp, Fp);
                dR[0] = Rp[0]; dR[1] = Rp[1];
                for (int q = 0; q < 2 * DIM; ++q) { dF[q][0] = Fp[q][0]; dF[q][1] = Fp[q][1]; }
            } else {
                dR[0] = R0[0]; dR[1] = R0[1];
                for (int q = 0; q < 2 * DIM; ++q) { dF[q][0] = F0[q][0]; dF[q][1] = F0[q][1]; }
            }
            if (method <= 0) {
                pri[pv] -= delta + eps;
                delta += eps;
                fd_local_residual<DIM>(P, col, h, ci, (pv == 0 ? FdState{pri[0], pri[1], base.pc, base.lw, base.ln} : fd_state<DIM>(P, P.law[li], pri[0], pri[1])), Ki, li, so, dt, x,
                                       perm, iq, Rp, Fp);
                dR[0] -= Rp[0]; dR[1] -= Rp[1];
                for (int q = 0; q < 2 * DIM; ++q) { dF[q][0] -= Fp[q][0]; dF[q][1] -= Fp[q][1]; }
            } else {
                dR[0] -= R0[0]; dR[1] -= R0[1];
                for (int q = 0; q < 2 * DIM; ++q) { dF[q][0] -= F0[q][0]; dF[q][1] -= F0[q][1]; }
            }
            // block entry [eq][pv]
            Jd[pv] = dR[0] / delta;
            Jd[2 + pv] = dR[1] / delta;
            for (int q = 0; q < 2 * DIM; ++q) {
                Jn[q][pv] = dF[q][0] / delta;
                Jn[q][2 + pv] = dF[q][1] / delta;
            }
        }
        store_block(J, N, 0, s, Jd);
#pragma unroll
        for (int axis = 0; axis < DIM; ++axis)
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int64_t sj = neighbour_split(P, col, h, ci, axis, side);
                if (sj >= 0) store_block(J, N, opposite_band(band_of(axis, side)), sj, Jn[2 * axis + side]);
            }
    }
    if (bad) atomicOr(flags, 1);
    block_max_publish(localMax, errmax);
}

// S_w = 1 state per region: p_cnw and k_r / mu of both phases for the free-flow boundary
// (out[0..5]), and the intensive quantities with their derivatives (out[6..17])
__global__ void k_boundary_constants(const __grid_constant__ Phys P, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int r = 0; r < 2; ++r) {
        MatOut m = material(P.law[r], 1.0);
        out[3 * r] = m.pc.v;
        out[3 * r + 1] = m.krw.v / P.mu[0];
        out[3 * r + 2] = m.krn.v / P.mu[1];
        const IqVals q = intensive_values_full(P, 1.0, r);
        const double v[6] = {q.pc, q.dpc, q.lw, q.dlw, q.ln, q.dln};
        for (int c = 0; c < 6; ++c) out[6 + 6 * r + c] = v[c];
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

cudaError_t boundary_constants(Phys& P, cudaStream_t stream) {
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(double) * 18);
    if (e != cudaSuccess) return e;
    k_boundary_constants<<<1, 32, 0, stream>>>(P, d);
    double h[18] = {0};
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    if (e != cudaSuccess) return e;
    for (int r = 0; r < 2; ++r) {
        P.bndPc[r] = h[3 * r];
        P.bndLam[r][0] = h[3 * r + 1];
        P.bndLam[r][1] = h[3 * r + 2];
        for (int c = 0; c < 6; ++c) P.sat1[r][c] = h[6 + 6 * r + c];
    }
    return cudaSuccess;
}

ewg_status compute_boundary_constants(ewg_ctx* ctx) {
    return cuda_fail(ctx, boundary_constants(ctx->P, ctx->stream), "boundary constants");
}

ewg_status launch_intensive(ewg_ctx* ctx, const double2* x) {
    int g1 = grid_size_for(ctx, (const void*)k_intensive, kLinBlock);
    EWG_LAUNCH(ctx, K_INTENSIVE, k_intensive, g1, kLinBlock, ctx->P, x, ctx->lens, ctx->iq);
    return cuda_fail(ctx, cudaGetLastError(), "k_intensive");
}

ewg_status launch_initial_solution(ewg_ctx* ctx, double2* x) {
    int grid = grid_size_for(ctx, (const void*)k_initial, kLinBlock);
    EWG_LAUNCH(ctx, K_INITIAL, k_initial, grid, kLinBlock, ctx->P, x);
    return cuda_fail(ctx, cudaGetLastError(), "k_initial");
}

void build_face_geo(const Phys& P, std::vector<FaceGeo>& geo) {
    const int n3[3] = {P.nx, P.ny, P.nz};
    geo.assign(2 * (n3[0] + n3[1] + n3[2]), FaceGeo{});
    for (int axis = 0; axis < 3; ++axis)
        for (int idx = 0; idx < n3[axis]; ++idx)
            for (int side = 0; side < 2; ++side) {
                // the operations of interior_face, in the same order
                const double h = P.h[axis];
                const int ia = idx + (axis == 2 ? P.kOrigin : 0);
                const double xc = (ia + 0.5) * h;
                const double xcj = (ia + (side ? 1 : -1) + 0.5) * h;
                const double dA = xcj - xc;
                const double distSq = dA * dA;
                FaceGeo G;
                G.coef = dA / distSq;
                G.dA = dA;
                G.gt[0] = G.gt[1] = 0.0;
                if (axis == 1) {
                    const double xf = (ia + side) * h;
                    const double gIn = -P.g * (xc - xf), gEx = -P.g * (xcj - xf);
                    for (int a = 0; a < 2; ++a) {
                        const double rho = P.rho[a];
                        const double pStatIn = -rho * gIn;
                        const double pStatEx = -(rho * gEx);
                        G.gt[a] = (pStatEx - pStatIn) / distSq;
                    }
                }
                geo[face_geo_index(n3, axis, idx, side)] = G;
            }
}

ewg_status build_interior_tables(ewg_ctx* ctx) {
    const Phys& P = ctx->P;
    if (P.dim != 3) return EWG_OK;
    std::vector<FaceGeo> geo;
    build_face_geo(P, geo);
    cudaError_t e;
    if ((e = cudaMalloc(&ctx->geo, sizeof(FaceGeo) * geo.size())) != cudaSuccess) return cuda_fail(ctx, e, "alloc face geometry");
    if ((e = cudaMemcpyAsync(ctx->geo, geo.data(), sizeof(FaceGeo) * geo.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "upload face geometry");
    // the host vector goes out of scope: finish the copy first
    return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync tables");
}

// resident blocks per SM the interior kernel is compiled for (register budget 65536 / (256 x it))
#ifndef EWG_INTERIOR_MIN_BLOCKS
#define EWG_INTERIOR_MIN_BLOCKS 2
#endif
constexpr int kInteriorMinBlocks = EWG_INTERIOR_MIN_BLOCKS;

template <typename JT, bool WITH_J>
static void launch_assemble3(ewg_ctx* ctx, double dt, const double2* x, double2* r, JT* J) {
    auto k = k_assemble3<JT, WITH_J, kInteriorMinBlocks>;
    int g = grid_size_for(ctx, (const void*)k, kAsm3Block);
    EWG_LAUNCH(ctx, K_ASSEMBLE, k, g, kAsm3Block, ctx->P, ctx->geo, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt,
               r, J, ctx->d_errmax, ctx->d_flags);
}

static ewg_status read_linearize_result(ewg_ctx* ctx, double* maxOut, int* nonfinite);

ewg_status launch_linearize(ewg_ctx* ctx, double dt, bool withJacobian, const double2* x,
                            double2* r, double* maxOut, int* nonfinite) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(ctx->d_errmax, 0, sizeof(unsigned long long), ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "memset errmax");
    if ((e = cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "memset flags");
    const bool three = ctx->P.dim == 3;
    const bool fd = withJacobian && ctx->localLinearizer == EWG_LOCAL_LINEARIZER_FD;
    int g1 = grid_size_for(ctx, (const void*)k_intensive, kLinBlock);
    EWG_LAUNCH(ctx, K_INTENSIVE, k_intensive, g1, kLinBlock, ctx->P, x, ctx->lens, ctx->iq);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "k_intensive");
    if (fd) {
        const int m = ctx->fdMethod;
        if (ctx->jacPrecision == EWG_PRECISION_MIXED) {
            auto k = three ? k_assemble_fd<3, float> : k_assemble_fd<2, float>;
            int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
            EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt,
                       ctx->refPressure, m, r, ctx->J32, ctx->d_errmax, ctx->d_flags);
        } else {
            auto k = three ? k_assemble_fd<3, double> : k_assemble_fd<2, double>;
            int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
            EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt,
                       ctx->refPressure, m, r, ctx->J, ctx->d_errmax, ctx->d_flags);
        }
    } else if (three) {
        if (!withJacobian)
            launch_assemble3<double, false>(ctx, dt, x, r, nullptr);
        else if (ctx->jacPrecision == EWG_PRECISION_MIXED)
            launch_assemble3<float, true>(ctx, dt, x, r, ctx->J32);
        else
            launch_assemble3<double, true>(ctx, dt, x, r, ctx->J);
    } else if (!withJacobian) {
        auto k = k_assemble<2, double, false>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                   nullptr, ctx->d_errmax, ctx->d_flags);
    } else if (ctx->jacPrecision == EWG_PRECISION_MIXED) {
        auto k = k_assemble<2, float, true>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                   ctx->J32, ctx->d_errmax, ctx->d_flags);
    } else {
        auto k = k_assemble<2, double, true>;
        int g2 = grid_size_for(ctx, (const void*)k, kLinBlock);
        EWG_LAUNCH(ctx, K_ASSEMBLE, k, g2, kLinBlock, ctx->P, x, ctx->sold, ctx->perm, ctx->lens, ctx->iq, dt, r,
                   ctx->J, ctx->d_errmax, ctx->d_flags);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "k_assemble");
    return read_linearize_result(ctx, maxOut, nonfinite);
}

// the residual max-norm and the non-finite flag of the last linearization, read back when asked
static ewg_status read_linearize_result(ewg_ctx* ctx, double* maxOut, int* nonfinite) {
    cudaError_t e;
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
