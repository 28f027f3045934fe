// Batched ensemble of 3D lens problems on one device (ewg_ensemble_* in include/ewg.h).
//
// The reference runs one lens problem per Simulator (tests/problems/lensproblem.hh with
// NewtonMethod::apply, nonlinear/newtonmethod.hh:308-517, and the step-halving retry of
// FvBaseProblem::timeIntegration, fvbaseproblem.hh:507-550). An ensemble of permeability
// realizations is many such runs; here all of them advance together in the same launches.
//
// Design
//   * Members are concatenated in flat arrays: member m owns cells [off_m, off_m + N_m) of every
//     per-cell vector (red-black split order inside the member, as for a single context) and the
//     plane blocks 6 off_m (intensive-quantity cache, stride N_m), 28 off_m (7 Jacobian bands),
//     4 off_m (inverted diagonal blocks) and 12 off_m (L factors of the black rows, stride N_m/2).
//   * Work is cut into tiles of kEnsTileH consecutive half indices of one member; a block of
//     kEnsTile threads works on one tile at a time (each thread a strided set of half indices:
//     both colours for cell kernels, one colour for the ILU sweeps). Every kernel is a persistent loop of resident blocks over the tile
//     table; tiles of members outside the current round (Newton finished, or BiCGStab stopped)
//     are skipped, so members of uneven size stop independently inside shared launches.
//   * BiCGStab state (bicgstabsolver.hh:116-326 with CombinedCriterion) is one BiState per
//     member. Each reduction ends per member: the tile that completes a member last sums that
//     member's tile partials in tile order (deterministic for a given tile table) and updates its
//     scalars.
//   * The nine kernels of a BiCGStab iteration are captured check_interval times over in one CUDA
//     graph that is replayed until no member is running.
//   * Launch shapes: the block is fixed (kEnsTile threads); an autotuner times, per kernel
//     class, the number of resident blocks (multiples of the SM count) and, for the assembly,
//     the register budget variant, and keeps the fastest. Sum reductions do not depend on the
//     launch shape, so results do not depend on the tuning.
//   * ILU(0) order: red-black, or the single problem's box-8-colour order (ewg_box8.cuh) when every
//     member's grid has it; the box-8 solve keeps each member's BiCGStab vectors in its box-8 order.
//   * Newton runs per member in supersteps: each superstep linearizes the members still iterating,
//     solves the ones that need a correction and updates them; a member whose step fails is
//     restored and restarts with half the step size. The decisions are taken either on the host
//     between supersteps (ewg_ensemble_advance) or on the device, with whole supersteps replayed by
//     a CUDA graph WHILE node (ewg_ensemble_advance_device).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ewg_assemble.cuh"
#include "ewg_box8.cuh"
#include "ewg_krylov.cuh"

namespace {
thread_local std::string g_ensCreateError;
}

namespace ewg {

constexpr int kEnsTile = 256;    // threads per block
// half indices per tile (8 per thread with 2048: the tile prologue is amortized; 1024 and 4096
// measured 4 % slower on the 64-member benchmark ensemble)
#ifndef EWG_ENS_TILE_H
#define EWG_ENS_TILE_H 2048
#endif
constexpr int kEnsTileH = EWG_ENS_TILE_H;
constexpr int kEnsBands = 7;   // 3D: diagonal + 6 faces
// resident blocks per SM the BiCGStab kernels are compiled for (register budgets 64 and 48)
constexpr int kEnsBlocksSpmv = 4;
constexpr int kEnsBlocksVec = 5;

struct EnsMember {
    Phys P;
    int64_t off;     // first cell of the member in the flat per-cell arrays
    int64_t geoOff;  // first entry of its face-geometry table
    int32_t tile0, ntiles;
};
static_assert(sizeof(EnsMember) % 8 == 0, "EnsMember is copied as 8-byte words");

enum EnsStatus { ST_IDLE = 5, ST_PENDING = 6 };

// kernel classes with their own launch shape
enum EnsClass {
    EC_INTENSIVE = 0, EC_ASSEMBLE, EC_FACTOR, EC_CELL, EC_ILU_BLACK, EC_ILU_RED, EC_SPMV_ALPHA,
    EC_SPMV_OMEGA, EC_P, EC_HS, EC_XR, EC_NUM
};

// ---- tile prologue ------------------------------------------------------------------------------

// Reads tile t, decides (once per block) whether its member takes part, and copies the member's
// descriptor into shared memory. Returns the member or -1; uniform across the block.
__device__ __forceinline__ int begin_tile(const EnsMember* __restrict__ mem, const int2* __restrict__ tiles, int t,
                                          const int* __restrict__ mask, const BiState* __restrict__ st, int want,
                                          EnsMember& sm, int* sh) {
    __syncthreads();  // the previous tile is done with sm and sh
    if (threadIdx.x == 0) {
        const int2 tl = tiles[t];
        bool act = true;
        if (mask) act = mask[tl.x] != 0;
        if (st) act = act && st[tl.x].status == want;
        sh[0] = act ? tl.x : -1;
        sh[1] = tl.y;
    }
    __syncthreads();
    const int m = sh[0];
    if (m < 0) return -1;
    const uint64_t* src = reinterpret_cast<const uint64_t*>(mem + m);
    uint64_t* dst = reinterpret_cast<uint64_t*>(&sm);
    for (int i = threadIdx.x; i < (int)(sizeof(EnsMember) / 8); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    return m;
}

__device__ __forceinline__ int64_t tile_end(const Phys& P, int64_t h0) {
    return h0 + kEnsTileH < P.Nh ? h0 + kEnsTileH : P.Nh;
}

// Block-wide max of non-negative doubles published with an integer atomicMax on the bit pattern.
__device__ __forceinline__ void block_max_atomic(double v, unsigned long long* out) {
    __shared__ double smax[kEnsTile / 32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) smax[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? smax[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0 && v > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

// Per-member deterministic reduction of NS sums and NM maxima. Every tile of the member calls it
// once; the tile that arrives last sums the member's tile partials in tile order and returns true
// (out valid in thread 0).
template <int NS, int NM>
__device__ __forceinline__ bool member_reduce(double (&v)[NS + NM], int tileIdx, int tile0, int ntiles,
                                              double* partials, unsigned* counter, double (&out)[NS + NM]) {
    constexpr int NV = NS + NM;
    __shared__ double sh[NV][kEnsTile / 32];
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
            partials[(size_t)tileIdx * NV + k] = a;
        }
        __threadfence();
        amLast = atomicAdd(counter, 1u) == (unsigned)(ntiles - 1);
    }
    __syncthreads();
    if (!amLast) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < ntiles; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double u = __ldcg(&partials[(size_t)(tile0 + b) * NV + k]);
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

// the tile list and its length live on the device, so a captured launch follows list updates
#define ENS_ARGS const EnsMember *__restrict__ mem, const int2 *__restrict__ tiles, const int *__restrict__ nTilesPtr
#define ENS_TILE_LOOP for (int t = blockIdx.x, nT_ = *nTilesPtr; t < nT_; t += gridDim.x)

// ---- state and linearization kernels ------------------------------------------------------------

// mode 0: hydrostatic initial state into x0 and x1 (LensProblem::initial, lensproblem.hh:545-578)
// mode 1: x1 = x0 (advanceTimeLevel)   mode 2: x0 = x1 (updateFailed)   mode 3: levels unchanged
// every mode ends with sold = storage(x1) (the storage cache of the old time level)
__global__ void __launch_bounds__(kEnsTile) ke_levels(ENS_ARGS, const int* __restrict__ mask, int mode,
                                                      double2* __restrict__ x0, double2* __restrict__ x1,
                                                      double2* __restrict__ sold) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        if (begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh) < 0) continue;
        const Phys& P = sm.P;
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                if (mode == 0) {
                    const CellIdx ci = cell_of(P, col, h);
                    const double y = (ci.j + 0.5) * P.h[1];
                    const double depth = P.L[1] - y;
                    const double densityW = P.rho[0];
                    const double2 v = make_double2(P.pRef - densityW * (-P.g) * depth, 1.0);
                    x0[s] = v;
                    x1[s] = v;
                } else if (mode == 1) {
                    x1[s] = x0[s];
                } else if (mode == 2) {
                    x0[s] = x1[s];
                }
                const double Sw = x1[s].y;
                sold[s] = make_double2(P.porosity * Sw * P.rho[0], P.porosity * (1.0 - (0.0 + Sw)) * P.rho[1]);
            }
        }
    }
}

__global__ void __launch_bounds__(kEnsTile) ke_intensive(ENS_ARGS, const int* __restrict__ mask,
                                                         const double2* __restrict__ x,
                                                         const uint8_t* __restrict__ lens, double* __restrict__ iq) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        if (begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh) < 0) continue;
        const Phys& P = sm.P;
        const int64_t off = sm.off;
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            intensive_cell(P, x + off, lens + off, iq + 6 * off, h, false);
            intensive_cell(P, x + off, lens + off, iq + 6 * off, P.Nh + h, false);
        }
    }
}

template <typename JT, bool WITH_J, int MINB>
__global__ void __launch_bounds__(kEnsTile, MINB) ke_assemble(
    ENS_ARGS, const int* __restrict__ mask, const FaceGeo* __restrict__ geo, const double* __restrict__ dtArr,
    const double2* __restrict__ x, const double2* __restrict__ sold, const double* __restrict__ perm,
    const uint8_t* __restrict__ lens, const double* __restrict__ iq, double2* __restrict__ r, JT* __restrict__ J,
    unsigned long long* __restrict__ errmax, int* __restrict__ flags) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh);
        if (m < 0) continue;
        const Phys& P = sm.P;
        const int64_t off = sm.off;
        const int64_t hEnd = tile_end(P, sh[1]);
        double mx = 0.0;
        int bad = 0;
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            const double dt = dtArr[m];
            for (int col = 0; col < 2; ++col)
                mx = fmax(mx, assemble_cell3<JT, WITH_J>(
                                  P, geo + sm.geoOff, x + off, sold + off, perm + off, lens + off, iq + 6 * off, dt,
                                  r + off, WITH_J ? J + kEnsBands * 4 * off : J, col * P.Nh + h, bad,
                                  nbr_global(x + off, perm + off, iq + 6 * off, P.N)));
        }
        if (bad) atomicOr(&flags[m], 1);
        block_max_atomic(mx, &errmax[m]);
    }
}

// x0 -= dx for the members in mask (newtonmethod.hh:743-809); a non-finite dx sets flags[m] bit 2
template <typename T, bool B8>
__global__ void __launch_bounds__(kEnsTile) ke_update(ENS_ARGS, const int* __restrict__ mask, double2* __restrict__ x0,
                                                      const typename V2T<T>::type* __restrict__ dx,
                                                      int* __restrict__ flags) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh);
        if (m < 0) continue;
        const Phys& P = sm.P;
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            int bad = 0;
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                const int64_t sx = B8 ? sm.off + b8_to_split_pos(P, col * P.Nh + h) : s;  // dx is in solver order
                const auto d = dx[s];
                const double d0 = (double)d.x, d1 = (double)d.y;
                if (!isfinite(d0) || !isfinite(d1)) bad = 1;
                double2 v = x0[sx];
                v.x -= d0;
                v.y -= d1;
                x0[sx] = v;
            }
            if (bad) atomicOr(&flags[m], 2);
        }
    }
}

// ---- preconditioner setup -----------------------------------------------------------------------

// red rows: Dinv = inv(A_rr); singular blocks set flags[m] bit 4
template <typename T>
__global__ void __launch_bounds__(kEnsTile) ke_diag_inverse_red(ENS_ARGS, const int* __restrict__ mask,
                                                                const T* __restrict__ J, T* __restrict__ Dinv,
                                                                int* __restrict__ flags) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh);
        if (m < 0) continue;
        const Phys& P = sm.P;
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            if (!diag_inverse_row(P.N, J + kEnsBands * 4 * sm.off, Dinv + 4 * sm.off, h)) atomicOr(&flags[m], 4);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kEnsTile) ke_ilu_black_factor(ENS_ARGS, const int* __restrict__ mask,
                                                                const T* __restrict__ J, T* __restrict__ Dinv,
                                                                T* __restrict__ L, int* __restrict__ flags) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh);
        if (m < 0) continue;
        const Phys& P = sm.P;
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            if (!ilu_black_factor_row(P, J + kEnsBands * 4 * sm.off, Dinv + 4 * sm.off, L + 12 * sm.off, h))
                atomicOr(&flags[m], 4);
        }
    }
}

// b = (T) r for the members in mask (B8: b in box-8 order)
template <typename T, bool B8>
__global__ void __launch_bounds__(kEnsTile) ke_rhs(ENS_ARGS, const int* __restrict__ mask, const double2* __restrict__ r,
                                                   typename V2T<T>::type* __restrict__ b) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        if (begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh) < 0) continue;
        const Phys& P = sm.P;
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                const double2 v = r[B8 ? sm.off + b8_to_split_pos(P, col * P.Nh + h) : s];
                typename V2T<T>::type o;
                o.x = (T)v.x;
                o.y = (T)v.y;
                b[s] = o;
            }
        }
    }
}

// BiCGStab state of the members in mask: the solver options and ST_PENDING (the init kernel starts
// them); other members keep their state, so members can start solves while others iterate
__global__ void ke_bicg_arm(const int* __restrict__ mask, int M, BiState tmpl, BiState* __restrict__ st) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M && mask[m]) st[m] = tmpl;
}

// ---- BiCGStab -------------------------------------------------------------------------------------

#define ENS_BICG_ARGS BiState *__restrict__ st, double *__restrict__ partials, unsigned *__restrict__ counters

template <typename T>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksVec) ke_bicg_init(ENS_ARGS, const typename V2T<T>::type* __restrict__ b,
                                                         typename V2T<T>::type* __restrict__ x,
                                                         typename V2T<T>::type* __restrict__ r,
                                                         typename V2T<T>::type* __restrict__ r0,
                                                         typename V2T<T>::type* __restrict__ v,
                                                         typename V2T<T>::type* __restrict__ p, ENS_BICG_ARGS) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_PENDING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        double red[2] = {0.0, 0.0};  // sum b.b, max |b|
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x)
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                const auto bs = b[s];
                typename V2T<T>::type z;
                z.x = (T)0;
                z.y = (T)0;
                x[s] = z; v[s] = z; p[s] = z;
                r[s] = bs; r0[s] = bs;
                const double b0 = (double)bs.x, b1 = (double)bs.y;
                red[0] += b0 * b0 + b1 * b1;
                red[1] = fmax(red[1], fmax(absn(b0), absn(b1)));
            }
        double out[2];
        if (member_reduce<1, 1>(red, sm.tile0 + sh[1] / kEnsTileH, sm.tile0, sm.ntiles, partials, &counters[m], out) && threadIdx.x == 0) {
            BiState* s = st + m;
            s->resErr = fmax(out[1], DBL_MIN * 1e10);
            s->initResErr = s->resErr;
            s->lastResErr = s->resErr;
            s->stagnates = 0;
            s->iter = 0;
            s->restarts = 0;
            s->restartPending = 0;
            s->rho = 1.0; s->alpha = 1.0; s->omega = 1.0;
            s->r0r0 = out[0];
            s->status = ST_RUNNING;
            const double rel = s->resErr / fmax(1e-20, s->initResErr);
            if (rel <= s->relTol || s->resErr <= s->absTol) { s->status = ST_CONVERGED; continue; }
            iteration_top(s, out[0], out[0]);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksVec) ke_bicg_p(ENS_ARGS, const typename V2T<T>::type* __restrict__ r,
                                                      typename V2T<T>::type* __restrict__ r0,
                                                      typename V2T<T>::type* __restrict__ v,
                                                      typename V2T<T>::type* __restrict__ p,
                                                      const BiState* __restrict__ st) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            const bool restart = st[m].restartPending != 0;
            const double beta = st[m].beta, omega = st[m].omega;
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                const auto rs = r[s];
                typename V2T<T>::type vs = v[s], ps = p[s];
                if (restart) {
                    r0[s] = rs;
                    vs.x = (T)0; vs.y = (T)0;
                    ps = vs;
                    v[s] = vs;
                }
                double t0 = (double)vs.x * omega, t1 = (double)vs.y * omega;
                t0 -= (double)ps.x; t1 -= (double)ps.y;
                t0 *= -beta; t1 *= -beta;
                typename V2T<T>::type o;
                o.x = (T)((double)rs.x + t0);
                o.y = (T)((double)rs.y + t1);
                p[s] = o;
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksVec) ke_ilu_black_apply(ENS_ARGS, const T* __restrict__ Dinv, const T* __restrict__ L,
                                                               const typename V2T<T>::type* __restrict__ d,
                                                               typename V2T<T>::type* __restrict__ y,
                                                               const BiState* __restrict__ st) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            const int64_t off = sm.off;
            ilu_black_apply_row<T, T>(P, Dinv + 4 * off, L + 12 * off, d + off, y + off, st[m].w, h);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksVec) ke_ilu_red_apply(ENS_ARGS, const T* __restrict__ J, const T* __restrict__ Dinv,
                                                             const typename V2T<T>::type* __restrict__ d,
                                                             typename V2T<T>::type* __restrict__ y,
                                                             const BiState* __restrict__ st) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            const int64_t off = sm.off;
            const double w = st[m].w;
            ilu_red_apply_row<T, T>(P, J + kEnsBands * 4 * off, Dinv + 4 * off, d + off, y + off, w, 1.0 / w, h);
        }
    }
}

// v = A y; alpha = rho_i / (r0hat . v)
// B8: box-8 order, v = A y from the sweeps' intermediate w (spmv_row_b8_precond: J is the box-8
// copy A8, E8 = A_cc - D', W the forward sweep's output)
template <typename T, bool B8>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksSpmv) ke_spmv_alpha(ENS_ARGS, const T* __restrict__ J,
                                                          const typename V2T<T>::type* __restrict__ y,
                                                          const typename V2T<T>::type* __restrict__ r0,
                                                          typename V2T<T>::type* __restrict__ v,
                                                          const T* __restrict__ E8,
                                                          const typename V2T<T>::type* __restrict__ W, ENS_BICG_ARGS) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        const int64_t off = sm.off;
        double red[1] = {0.0};
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x)
            for (int col = 0; col < 2; ++col) {
                const int64_t s = col * P.Nh + h;
                double a0, a1;
                if (B8) spmv_row_b8_precond<T, T>(P, J + kEnsBands * 4 * off, E8 + 4 * off, W + off, st[m].w, y + off, s,
                                                  a0, a1);
                else spmv_row<T, T>(P, J + kEnsBands * 4 * off, y + off, s, a0, a1);
                typename V2T<T>::type o;
                o.x = (T)a0; o.y = (T)a1;
                v[off + s] = o;
                const auto rh = r0[off + s];
                red[0] += (double)rh.x * (double)o.x + (double)rh.y * (double)o.y;
            }
        double out[1];
        if (member_reduce<1, 0>(red, sm.tile0 + sh[1] / kEnsTileH, sm.tile0, sm.ntiles, partials, &counters[m], out) && threadIdx.x == 0) {
            BiState* s = st + m;
            const double breakdownEps = DBL_MIN * 1e10;
            s->restartPending = 0;
            const double denom = out[0];
            if (fabs(denom) <= breakdownEps) { s->status = ST_BREAKDOWN; continue; }
            s->alpha = s->rho_i / denom;
            if (fabs(s->alpha) <= breakdownEps) s->status = ST_BREAKDOWN;
        }
    }
}

// h = x + alpha y (in x), s = r - alpha v (in r); criterion on s with y as change indicator
template <typename T>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksVec) ke_hs(ENS_ARGS, typename V2T<T>::type* __restrict__ x,
                                                  const typename V2T<T>::type* __restrict__ y,
                                                  typename V2T<T>::type* __restrict__ r,
                                                  const typename V2T<T>::type* __restrict__ v, ENS_BICG_ARGS) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        const double alpha = st[m].alpha;
        double red[2] = {0.0, 0.0};  // max |s|, any y != 0
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x)
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                const auto ys = y[s], xs = x[s], rs = r[s], vs = v[s];
                typename V2T<T>::type hx, sx;
                hx.x = (T)((double)ys.x * alpha + (double)xs.x);
                hx.y = (T)((double)ys.y * alpha + (double)xs.y);
                sx.x = (T)((double)rs.x - (double)vs.x * alpha);
                sx.y = (T)((double)rs.y - (double)vs.y * alpha);
                x[s] = hx;
                r[s] = sx;
                red[0] = fmax(red[0], fmax(absn((double)sx.x), absn((double)sx.y)));
                if (ys.x != (T)0 || ys.y != (T)0) red[1] = 1.0;
            }
        double out[2];
        if (member_reduce<0, 2>(red, sm.tile0 + sh[1] / kEnsTileH, sm.tile0, sm.ntiles, partials, &counters[m], out) && threadIdx.x == 0) {
            BiState* s = st + m;
            s->lastResErr = s->resErr;
            s->resErr = out[0];
            s->stagnates = out[1] == 0.0;
            criterion_check(s);
        }
    }
}

// t = A z; omega = (t . s) / (t . t)
template <typename T, bool B8>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksSpmv) ke_spmv_omega(ENS_ARGS, const T* __restrict__ J,
                                                          const typename V2T<T>::type* __restrict__ z,
                                                          const typename V2T<T>::type* __restrict__ sres,
                                                          typename V2T<T>::type* __restrict__ tv,
                                                          const T* __restrict__ E8,
                                                          const typename V2T<T>::type* __restrict__ W, ENS_BICG_ARGS) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        const int64_t off = sm.off;
        double red[2] = {0.0, 0.0};
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x)
            for (int col = 0; col < 2; ++col) {
                const int64_t s = col * P.Nh + h;
                double a0, a1;
                if (B8) spmv_row_b8_precond<T, T>(P, J + kEnsBands * 4 * off, E8 + 4 * off, W + off, st[m].w, z + off, s,
                                                  a0, a1);
                else spmv_row<T, T>(P, J + kEnsBands * 4 * off, z + off, s, a0, a1);
                typename V2T<T>::type o;
                o.x = (T)a0; o.y = (T)a1;
                tv[off + s] = o;
                const auto ss = sres[off + s];
                const double t0 = (double)o.x, t1 = (double)o.y;
                red[0] += t0 * t0 + t1 * t1;
                red[1] += t0 * (double)ss.x + t1 * (double)ss.y;
            }
        double out[2];
        if (member_reduce<2, 0>(red, sm.tile0 + sh[1] / kEnsTileH, sm.tile0, sm.ntiles, partials, &counters[m], out) && threadIdx.x == 0) {
            BiState* s = st + m;
            const double breakdownEps = DBL_MIN * 1e10;
            if (fabs(out[0]) <= breakdownEps) { s->status = ST_BREAKDOWN; continue; }
            s->omega = out[1] / out[0];
            if (fabs(s->omega) <= breakdownEps) s->status = ST_BREAKDOWN;
        }
    }
}

// x += omega z; criterion on r (still s) with z as change indicator; r += -omega t; then the next
// iteration's r0hat . r and r . r
template <typename T>
__global__ void __launch_bounds__(kEnsTile, kEnsBlocksVec) ke_xr(ENS_ARGS, typename V2T<T>::type* __restrict__ x,
                                                  const typename V2T<T>::type* __restrict__ z,
                                                  typename V2T<T>::type* __restrict__ r,
                                                  const typename V2T<T>::type* __restrict__ tv,
                                                  const typename V2T<T>::type* __restrict__ r0, ENS_BICG_ARGS) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;  // the fields the rows use, in registers
        const int64_t hEnd = tile_end(P, sh[1]);
        const double omega = st[m].omega;
        double red[4] = {0.0, 0.0, 0.0, 0.0};  // sum r0.r', sum r'.r', max |s|, any z != 0
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x)
            for (int col = 0; col < 2; ++col) {
                const int64_t s = sm.off + col * P.Nh + h;
                const auto xs = x[s], zs = z[s], rs = r[s], ts = tv[s], rh = r0[s];
                typename V2T<T>::type xn, rn;
                xn.x = (T)((double)xs.x + omega * (double)zs.x);
                xn.y = (T)((double)xs.y + omega * (double)zs.y);
                x[s] = xn;
                red[2] = fmax(red[2], fmax(absn((double)rs.x), absn((double)rs.y)));
                if (zs.x != (T)0 || zs.y != (T)0) red[3] = 1.0;
                rn.x = (T)((double)rs.x + (-omega) * (double)ts.x);
                rn.y = (T)((double)rs.y + (-omega) * (double)ts.y);
                r[s] = rn;
                const double r0v = (double)rn.x, r1v = (double)rn.y;
                red[0] += (double)rh.x * r0v + (double)rh.y * r1v;
                red[1] += r0v * r0v + r1v * r1v;
            }
        double out[4];
        if (member_reduce<2, 2>(red, sm.tile0 + sh[1] / kEnsTileH, sm.tile0, sm.ntiles, partials, &counters[m], out) && threadIdx.x == 0) {
            BiState* s = st + m;
            s->lastResErr = s->resErr;
            s->resErr = out[2];
            s->stagnates = out[3] == 0.0;
            criterion_check(s);
            if (s->status != ST_RUNNING) continue;
            s->iter += 1;
            iteration_top(s, out[0], out[1]);
        }
    }
}

// ---- box-8-colour ILU(0) for ensembles whose members all have that order -------------------------
//
// The single-problem box-8 factorization and sweeps (ewg_box8.cuh) per member: each member's
// Jacobian is copied into its box-8 order (stride N_m, the member's block of planes), and during
// the solve every BiCGStab vector of a member is in that order (the right-hand side is converted
// on the way in, the correction on the way out). A tile of kEnsTileH half indices of a member is
// kEnsTileH / 32 superblocks of it, so the sweeps take a tile as kEnsTileH / 1024 blocks of 32
// boxes and the factorization as one thread per superblock.

constexpr int kEnsB8Sub = kEnsTileH / 1024;  // 32-box sub-tiles of a tile

// A8 = J in box-8 order, block-packed (7 bands of 2x2 blocks per member)
template <typename T>
__global__ void __launch_bounds__(kEnsTile) ke_b8_matrix(ENS_ARGS, const int* __restrict__ mask, const T* __restrict__ J,
                                                         T* __restrict__ A8) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    ENS_TILE_LOOP {
        if (begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh) < 0) continue;
        const Phys P = sm.P;
        const int64_t hEnd = tile_end(P, sh[1]);
        const T* Jm = J + kEnsBands * 4 * sm.off;
        T* Am = A8 + kEnsBands * 4 * sm.off;
        // half index h -> the pair of cells two apart in x (colour bit 0 clear / set, same place and
        // box), neighbours in the split order: aligned pair loads, packed block stores
        const typename V2T<T>::type* __restrict__ Jm2 = reinterpret_cast<const typename V2T<T>::type*>(Jm);
        for (int64_t h = sh[1] + threadIdx.x; h < hEnd; h += blockDim.x) {
            const int64_t gi = h / P.Nb, b = h - gi * P.Nb;
            const int64_t g = ((gi >> 3) << 4) | (gi & 7);
            const int64_t s8 = g * P.Nb + b, s8b = s8 + 8 * P.Nb;
            const int64_t sp = b8_to_split_pos(P, s8);  // even; s8b sits at sp + 1
            for (int band = 0; band < kEnsBands; ++band) {
                double v[4], w[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const typename V2T<T>::type a = Jm2[((int64_t)(4 * band + c) * P.N + sp) >> 1];
                    v[c] = (double)a.x;
                    w[c] = (double)a.y;
                }
                store_pb(Am, P.N, band, s8, v);
                store_pb(Am, P.N, band, s8b, w);
            }
        }
    }
}

// factorization of one colour level: one thread per superblock of the tile and colour of the level;
// a singular pivot sets bit 4
template <typename T, int LEVEL>
__global__ void __launch_bounds__(kEnsTile) ke_b8_factor(ENS_ARGS, const int* __restrict__ mask, const T* __restrict__ A8,
                                                         T* __restrict__ Dinv8, T* __restrict__ L8, T* __restrict__ E8,
                                                         int* __restrict__ flags) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    constexpr int NC = B8Level<LEVEL>::count;
    static_assert(NC * (kEnsTileH / 32) <= kEnsTile, "one thread per (superblock, colour) of a tile");
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, mask, nullptr, 0, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;
        const int ci = threadIdx.x / (kEnsTileH / 32);
        const int64_t b = sh[1] / 32 + threadIdx.x % (kEnsTileH / 32);
        if (ci >= NC || b >= P.Nb) continue;
        const int64_t off = sm.off;
        const T* A = A8 + kEnsBands * 4 * off;
        T* Di = Dinv8 + 4 * off;
        T* L = L8 + 24 * off;
        T* E = E8 + 4 * off;
        bool ok = true;
#define EWG_B8_CALL(C) ok = b8_factor_box<T, C>(P, A, Di, L, E, b)
        EWG_B8_LEVEL_DISPATCH(LEVEL, ci, EWG_B8_CALL);
#undef EWG_B8_CALL
        if (!ok) atomicOr(&flags[m], 4);
    }
}

// forward sweep of one colour level for the running members: w = (D' + L_A)^-1 d on its cells
template <typename T, int LEVEL>
__global__ void __launch_bounds__(kEnsTile, sizeof(T) == 4 ? kEnsBlocksSpmv + 2 : kEnsBlocksSpmv) ke_b8_forward(ENS_ARGS, const T* __restrict__ L8,
                                                                          const typename V2T<T>::type* __restrict__ d,
                                                                          typename V2T<T>::type* __restrict__ w,
                                                                          const BiState* __restrict__ st) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    __shared__ double2 SB[2][8][32];
    constexpr int NC = B8Level<LEVEL>::count;
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    int k = 0;
    ENS_TILE_LOOP {
        if (begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh) < 0) continue;
        const Phys P = sm.P;
        const int64_t off = sm.off;
        for (int ci = 0; ci < NC; ++ci)
            for (int sub = 0; sub < kEnsB8Sub; ++sub, ++k) {
#define EWG_B8_CALL(C) \
    b8_forward_tile<T, T, C>(P, L8 + 24 * off, d + off, w + off, sh[1] / 32 + sub * 32, SB[k & 1], lane, q)
                EWG_B8_LEVEL_DISPATCH(LEVEL, ci, EWG_B8_CALL);
#undef EWG_B8_CALL
            }
    }
}

// backward sweep of one colour level: y = relax (D')^-1 (w - U_A y / relax) on its cells
template <typename T, int LEVEL>
__global__ void __launch_bounds__(kEnsTile, sizeof(T) == 4 ? kEnsBlocksSpmv + 2 : kEnsBlocksSpmv) ke_b8_backward(ENS_ARGS, const T* __restrict__ A8,
                                                                           const T* __restrict__ Dinv8,
                                                                           const typename V2T<T>::type* __restrict__ wv,
                                                                           typename V2T<T>::type* __restrict__ y,
                                                                           const BiState* __restrict__ st) {
    __shared__ EnsMember sm;
    __shared__ int sh[2];
    __shared__ double2 SB[2][8][32];
    constexpr int NC = B8Level<LEVEL>::count;
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    int k = 0;
    ENS_TILE_LOOP {
        const int m = begin_tile(mem, tiles, t, nullptr, st, ST_RUNNING, sm, sh);
        if (m < 0) continue;
        const Phys P = sm.P;
        const int64_t off = sm.off;
        const double w = st[m].w;
        for (int ci = 0; ci < NC; ++ci)
            for (int sub = 0; sub < kEnsB8Sub; ++sub, ++k) {
#define EWG_B8_CALL(C)                                                                                      \
    b8_backward_tile<T, T, C>(P, A8 + kEnsBands * 4 * off, Dinv8 + 4 * off, wv + off, y + off, w, 1.0 / w, \
                              sh[1] / 32 + sub * 32, SB[k & 1], lane, q)
                EWG_B8_LEVEL_DISPATCH(LEVEL, ci, EWG_B8_CALL);
#undef EWG_B8_CALL
            }
    }
}

// state of the device scheduler (ewg_ensemble_advance_device)
struct RunD {  // MemberRun on the device
    int phase, numIt;
    double error, lastError, dt0, h;
    int stepsLeft, halvingsStep, lastStatus, newton, linear, halvings;
    int fail, accept;  // the member's failed / accepted entry, cleared by the next settle
};

struct SchedD {
    long long supersteps;  // supersteps run so far
    long long limit;       // the WHILE loop stops after this many (set by the host per launch)
    int active;            // a member is linearizing or solving
    int error;             // EWG_ERR_TIMEOUT: a member's BiCGStab never left running
    int rounds;            // supersteps that linearized a member
    int linearIterations;
    double cellIterations;  // sums of integers below 2^53: exact in any order
};

struct NewtonD {
    double tol, maxError;
    int maxIt;
};

}  // namespace ewg

// ---- host side ----------------------------------------------------------------------------------

using namespace ewg;

struct ewg_ensemble {
    int M = 0;
    int device = 0;
    int numSMs = 148;
    int precision = EWG_PRECISION_MIXED;
    bool useGraph = true;
    int checkInterval = 8;
    int maxDiv = 10;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t tev[2] = {nullptr, nullptr};
    cudaEvent_t maskEv = nullptr;  // recorded after each upload from hMask
    std::string err;
    std::vector<EnsMember> hm;
    std::vector<int2> hTiles;
    int64_t total = 0;
    // device
    EnsMember* dm = nullptr;
    int nTiles = 0;
    double2 *x0 = nullptr, *x1 = nullptr, *sold = nullptr, *r = nullptr, *stage = nullptr;
    double* perm = nullptr;
    uint8_t* lens = nullptr;
    double* iq = nullptr;
    FaceGeo* geo = nullptr;
    void *J = nullptr, *Dinv = nullptr, *L = nullptr;
    void *kx = nullptr, *kr = nullptr, *kr0 = nullptr, *kv = nullptr, *kp = nullptr, *ky = nullptr, *kz = nullptr,
         *kb = nullptr;
    double* partials = nullptr;
    unsigned* counters = nullptr;
    BiState* st = nullptr;
    BiState* stSave = nullptr;
    int* mask = nullptr;
    unsigned long long* errmax = nullptr;
    int* flags = nullptr;      // linearization: bit 1 non-finite residual
    int* flagsF = nullptr;     // preconditioner setup: bit 4 singular diagonal block
    int* flagsU = nullptr;     // Newton update: bit 2 non-finite correction
    double* dtArr = nullptr;
    // pinned host mirrors
    BiState* hSt = nullptr;
    int* hMask = nullptr;
    unsigned long long* hErr = nullptr;
    int* hFlags = nullptr;
    int* hFlagsF = nullptr;
    int* hFlagsU = nullptr;
    double* hDt = nullptr;
    // launch shapes
    int grid[EC_NUM] = {};
    int asmVariant = 3;  // register budget: resident blocks per SM the assembly is compiled for
    bool tuned = false;
    // compact tile lists: A for the masked phases, B for the BiCGStab iterations (the graph reads B)
    struct TileList {
        int2* d = nullptr;
        int* dn = nullptr;
        int2* h = nullptr;     // pinned staging
        int* hn = nullptr;
        cudaEvent_t ev = nullptr;  // recorded after the last upload from h
    } tlA, tlB;
    // BiCGStab chunk graph
    cudaGraphExec_t graphExec = nullptr;
    double relaxation = 1.0;
    // box-8-colour ILU(0) (every member's grid has the order): the solve runs in box-8 order
    bool b8 = false;
    bool b8ok = false;         // every member has the order
    void *A8 = nullptr, *L8 = nullptr, *Dinv8 = nullptr, *E8 = nullptr, *W8 = nullptr;
    // device scheduler of ewg_ensemble_advance_device (allocated on its first call)
    ewg::RunD* dRun = nullptr;
    ewg::SchedD* dSched = nullptr;
    int* dPrefix = nullptr;
    int2* dTilesAll = nullptr;
    int *maskF = nullptr, *maskA = nullptr, *maskS = nullptr;
    ewg::RunD* hRun = nullptr;
    ewg::SchedD* hSched = nullptr;
};

namespace {

ewg_status ens_fail(ewg_ensemble* e, cudaError_t c, const char* what) {
    if (c == cudaSuccess) return EWG_OK;
    e->err = std::string(what) + ": " + cudaGetErrorString(c);
    return EWG_ERR_CUDA;
}

template <typename T>
using VT = typename V2T<T>::type;

template <typename T>
struct Ops {
    static VT<T>* v(void* p) { return (VT<T>*)p; }
    static T* m(void* p) { return (T*)p; }

    static void assemble(ewg_ensemble* e, bool withJ) {
        const int g = e->grid[EC_ASSEMBLE];
        if (!withJ) {
            ke_assemble<T, false, 3><<<g, kEnsTile, 0, e->stream>>>(
                e->dm, e->tlA.d, e->tlA.dn, e->mask, e->geo, e->dtArr, e->x0, e->sold, e->perm, e->lens, e->iq, e->r,
                (T*)nullptr, e->errmax, e->flags);
        } else if (e->asmVariant == 2) {
            ke_assemble<T, true, 2><<<g, kEnsTile, 0, e->stream>>>(
                e->dm, e->tlA.d, e->tlA.dn, e->mask, e->geo, e->dtArr, e->x0, e->sold, e->perm, e->lens, e->iq, e->r,
                m(e->J), e->errmax, e->flags);
        } else {
            ke_assemble<T, true, 3><<<g, kEnsTile, 0, e->stream>>>(
                e->dm, e->tlA.d, e->tlA.dn, e->mask, e->geo, e->dtArr, e->x0, e->sold, e->perm, e->lens, e->iq, e->r,
                m(e->J), e->errmax, e->flags);
        }
    }
    static void intensive(ewg_ensemble* e) {
        ke_intensive<<<e->grid[EC_INTENSIVE], kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, e->x0,
                                                                        e->lens, e->iq);
    }
    template <int LEVEL>
    static void b8_factor_level(ewg_ensemble* e, int g) {
        ke_b8_factor<T, LEVEL><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, m(e->A8),
                                                             m(e->Dinv8), m(e->L8), m(e->E8), e->flagsF);
    }
    static void factor(ewg_ensemble* e) {
        const int g = e->grid[EC_FACTOR];
        if (e->b8) {
            ke_b8_matrix<T><<<e->grid[EC_CELL], kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, m(e->J),
                                                                         m(e->A8));
            b8_factor_level<0>(e, g);
            b8_factor_level<1>(e, g);
            b8_factor_level<2>(e, g);
            b8_factor_level<3>(e, g);
            return;
        }
        ke_diag_inverse_red<T><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, m(e->J), m(e->Dinv),
                                                             e->flagsF);
        ke_ilu_black_factor<T><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, m(e->J), m(e->Dinv),
                                                             m(e->L), e->flagsF);
    }
    // box-8 sweeps of all colour levels for the running members: W = forward(d), y = backward(W)
    template <int C>
    static void b8_fwd(ewg_ensemble* e, int g, const VT<T>* d) {
        ke_b8_forward<T, C><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlB.d, e->tlB.dn, m(e->L8), d, v(e->W8), e->st);
    }
    template <int C>
    static void b8_bwd(ewg_ensemble* e, int g, VT<T>* y) {
        ke_b8_backward<T, C><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlB.d, e->tlB.dn, m(e->A8), m(e->Dinv8), v(e->W8), y,
                                                           e->st);
    }
    static void rhs_init(ewg_ensemble* e) {
        const int g = e->grid[EC_CELL];
        if (e->b8) ke_rhs<T, true><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, e->r, v(e->kb));
        else ke_rhs<T, false><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, e->r, v(e->kb));
        ke_bicg_init<T><<<g, kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, v(e->kb), v(e->kx), v(e->kr),
                                                      v(e->kr0), v(e->kv), v(e->kp), e->st, e->partials, e->counters);
    }
    // one kernel of the iteration by class (the autotuner times them one at a time)
    static void kernel(ewg_ensemble* e, int cls, int which) {
        const int g = e->grid[cls];
        auto* E = e;
        switch (cls) {
            case EC_P:
                ke_bicg_p<T><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, v(E->kr), v(E->kr0), v(E->kv),
                                                           v(E->kp), E->st);
                break;
            case EC_ILU_BLACK:
                if (E->b8) {  // the forward sweeps (d = p or s, into W)
                    const VT<T>* d = which ? v(E->kr) : v(E->kp);
                    b8_fwd<0>(E, g, d); b8_fwd<1>(E, g, d); b8_fwd<2>(E, g, d); b8_fwd<3>(E, g, d);
                    break;
                }
                ke_ilu_black_apply<T><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, m(E->Dinv), m(E->L),
                                                                    which ? v(E->kr) : v(E->kp),
                                                                    which ? v(E->kz) : v(E->ky), E->st);
                break;
            case EC_ILU_RED:
                if (E->b8) {  // the backward sweeps (from W into y or z)
                    VT<T>* y = which ? v(E->kz) : v(E->ky);
                    b8_bwd<3>(E, g, y); b8_bwd<2>(E, g, y); b8_bwd<1>(E, g, y); b8_bwd<0>(E, g, y);
                    break;
                }
                ke_ilu_red_apply<T><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, m(E->J), m(E->Dinv),
                                                                  which ? v(E->kr) : v(E->kp),
                                                                  which ? v(E->kz) : v(E->ky), E->st);
                break;
            case EC_SPMV_ALPHA:
                if (E->b8)
                    ke_spmv_alpha<T, true><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, m(E->A8), v(E->ky),
                                                                         v(E->kr0), v(E->kv), m(E->E8), v(E->W8), E->st,
                                                                         E->partials, E->counters);
                else
                    ke_spmv_alpha<T, false><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, m(E->J), v(E->ky),
                                                                          v(E->kr0), v(E->kv), nullptr, nullptr, E->st,
                                                                          E->partials, E->counters);
                break;
            case EC_HS:
                ke_hs<T><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, v(E->kx), v(E->ky), v(E->kr),
                                                       v(E->kv), E->st, E->partials, E->counters);
                break;
            case EC_SPMV_OMEGA:
                // t is stored in y (free after h)
                if (E->b8)
                    ke_spmv_omega<T, true><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, m(E->A8), v(E->kz),
                                                                         v(E->kr), v(E->ky), m(E->E8), v(E->W8), E->st,
                                                                         E->partials, E->counters);
                else
                    ke_spmv_omega<T, false><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, m(E->J), v(E->kz),
                                                                          v(E->kr), v(E->ky), nullptr, nullptr, E->st,
                                                                          E->partials, E->counters);
                break;
            case EC_XR:
                ke_xr<T><<<g, kEnsTile, 0, E->stream>>>(E->dm, E->tlB.d, E->tlB.dn, v(E->kx), v(E->kz), v(E->kr),
                                                       v(E->ky), v(E->kr0), E->st, E->partials, E->counters);
                break;
            default:
                break;
        }
    }
    static void iteration(ewg_ensemble* e) {
        kernel(e, EC_P, 0);
        kernel(e, EC_ILU_BLACK, 0);
        kernel(e, EC_ILU_RED, 0);
        kernel(e, EC_SPMV_ALPHA, 0);
        kernel(e, EC_HS, 0);
        kernel(e, EC_ILU_BLACK, 1);
        kernel(e, EC_ILU_RED, 1);
        kernel(e, EC_SPMV_OMEGA, 0);
        kernel(e, EC_XR, 0);
    }
    static void update(ewg_ensemble* e) {
        if (e->b8)
            ke_update<T, true><<<e->grid[EC_CELL], kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, e->x0,
                                                                            v(e->kx), e->flagsU);
        else
            ke_update<T, false><<<e->grid[EC_CELL], kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, e->x0,
                                                                             v(e->kx), e->flagsU);
    }
};

int resident_blocks(const void* k) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kEnsTile, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

// default launch shapes: every resident block once (persistent)
template <typename T>
void default_grids(ewg_ensemble* e) {
    const void* ks[EC_NUM] = {
        (const void*)ke_intensive, (const void*)ke_assemble<T, true, 3>, (const void*)ke_ilu_black_factor<T>,
        (const void*)ke_bicg_init<T>, (const void*)ke_ilu_black_apply<T>, (const void*)ke_ilu_red_apply<T>,
        (const void*)ke_spmv_alpha<T, false>, (const void*)ke_spmv_omega<T, false>, (const void*)ke_bicg_p<T>, (const void*)ke_hs<T>,
        (const void*)ke_xr<T>};
    for (int c = 0; c < EC_NUM; ++c) {
        int g = e->numSMs * resident_blocks(ks[c]);
        e->grid[c] = std::max(1, std::min(g, e->nTiles));
    }
}

ewg_status sync_read(ewg_ensemble* e, void* dst, const void* src, size_t bytes, const char* what) {
    cudaError_t c = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, e->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
    return ens_fail(e, c, what);
}

// The tiles of the members in `set` (in member order) into a device tile list. The pinned staging
// buffer is rewritten only after the previous upload from it has executed.
ewg_status set_tiles(ewg_ensemble* e, ewg_ensemble::TileList& tl, const std::vector<int>& set) {
    cudaError_t c = cudaEventSynchronize(tl.ev);
    if (c != cudaSuccess) return ens_fail(e, c, "wait tile upload");
    std::vector<int> ms(set);
    std::sort(ms.begin(), ms.end());
    int n = 0;
    for (int m : ms) {
        const EnsMember& em = e->hm[m];
        for (int k = 0; k < em.ntiles; ++k) tl.h[n++] = e->hTiles[em.tile0 + k];
    }
    *tl.hn = n;
    c = cudaMemcpyAsync(tl.dn, tl.hn, sizeof(int), cudaMemcpyHostToDevice, e->stream);
    if (c == cudaSuccess && n > 0) c = cudaMemcpyAsync(tl.d, tl.h, sizeof(int2) * n, cudaMemcpyHostToDevice, e->stream);
    if (c == cudaSuccess) c = cudaEventRecord(tl.ev, e->stream);
    return ens_fail(e, c, "upload tiles");
}

// Members of `set` take part in the next masked launches: the member mask and tile list A. The
// pinned host mask is rewritten only after the previous upload from it has executed.
ewg_status upload_mask(ewg_ensemble* e, const std::vector<int>& set) {
    cudaError_t c = cudaEventSynchronize(e->maskEv);
    if (c != cudaSuccess) return ens_fail(e, c, "wait mask upload");
    for (int m = 0; m < e->M; ++m) e->hMask[m] = 0;
    for (int m : set) e->hMask[m] = 1;
    c = cudaMemcpyAsync(e->mask, e->hMask, sizeof(int) * e->M, cudaMemcpyHostToDevice, e->stream);
    if (c == cudaSuccess) c = cudaEventRecord(e->maskEv, e->stream);
    if (c != cudaSuccess) return ens_fail(e, c, "upload mask");
    return set_tiles(e, e->tlA, set);
}

ewg_status levels(ewg_ensemble* e, const std::vector<int>& set, int mode) {
    if (set.empty()) return EWG_OK;
    ewg_status s = upload_mask(e, set);
    if (s) return s;
    ke_levels<<<e->grid[EC_CELL], kEnsTile, 0, e->stream>>>(e->dm, e->tlA.d, e->tlA.dn, e->mask, mode, e->x0, e->x1,
                                                           e->sold);
    return ens_fail(e, cudaGetLastError(), "levels");
}

// linearize the members of `set` at x0 with step sizes hDt; errors and flags into hErr / hFlags
template <typename T>
ewg_status linearize_set(ewg_ensemble* e, const std::vector<int>& set, bool withJ) {
    ewg_status s = upload_mask(e, set);
    if (s) return s;
    cudaError_t c;
    if ((c = cudaMemcpyAsync(e->dtArr, e->hDt, sizeof(double) * e->M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "upload dt");
    if ((c = cudaMemsetAsync(e->errmax, 0, sizeof(unsigned long long) * e->M, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "zero errmax");
    if ((c = cudaMemsetAsync(e->flags, 0, sizeof(int) * e->M, e->stream)) != cudaSuccess) return ens_fail(e, c, "zero flags");
    Ops<T>::intensive(e);
    Ops<T>::assemble(e, withJ);
    if ((c = cudaGetLastError()) != cudaSuccess) return ens_fail(e, c, "linearize");
    if ((c = cudaMemcpyAsync(e->hErr, e->errmax, sizeof(unsigned long long) * e->M, cudaMemcpyDeviceToHost, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "read errmax");
    return sync_read(e, e->hFlags, e->flags, sizeof(int) * e->M, "read flags");
}

double err_of(const ewg_ensemble* e, int m) {
    double v;
    memcpy(&v, &e->hErr[m], sizeof(v));
    return v;
}

template <typename T>
ewg_status build_graph(ewg_ensemble* e) {
    if (e->graphExec) return EWG_OK;
    cudaGraph_t g = nullptr;
    cudaError_t c = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (c != cudaSuccess) return ens_fail(e, c, "begin capture");
    for (int k = 0; k < e->checkInterval; ++k) Ops<T>::iteration(e);
    c = cudaStreamEndCapture(e->stream, &g);
    if (c != cudaSuccess) return ens_fail(e, c, "end capture");
    c = cudaGraphInstantiate(&e->graphExec, g, 0);
    cudaGraphDestroy(g);
    return ens_fail(e, c, "instantiate graph");
}

// The ILU(0) order of the solves: box-8-colour when every member's grid has it (ilu_ordering AUTO or
// BOX8; BOX8 on an ensemble where some member lacks it is an error), else red-black. A change of
// order drops the captured BiCGStab graph; the box-8 copies of the matrix are allocated on first use.
ewg_status ens_set_order(ewg_ensemble* e, const ewg_solve_opts* o) {
    if (o->ilu_ordering == EWG_ILU_ORDER_BOX8 && !e->b8ok) {
        e->err = "box-8 ILU ordering needs every member's nx, ny, nz to be multiples of 4";
        return EWG_ERR_INVALID;
    }
    const bool want = e->b8ok && (o->ilu_ordering == EWG_ILU_ORDER_AUTO || o->ilu_ordering == EWG_ILU_ORDER_BOX8);
    if (want && !e->A8) {
        const size_t sT = e->precision == EWG_PRECISION_MIXED ? sizeof(float) : sizeof(double);
        const int64_t n = e->total;
        cudaError_t c = cudaMalloc(&e->A8, sT * kEnsBands * 4 * n);
        if (c == cudaSuccess) c = cudaMalloc(&e->L8, sT * 24 * n);
        if (c == cudaSuccess) c = cudaMalloc(&e->Dinv8, sT * 4 * n);
        if (c == cudaSuccess) c = cudaMalloc(&e->E8, sT * 4 * n);
        if (c == cudaSuccess) c = cudaMalloc(&e->W8, sT * 2 * n);
        if (c != cudaSuccess) return ens_fail(e, c, "allocate box-8 ILU");
    }
    if (want != e->b8 && e->graphExec) {
        cudaGraphExecDestroy(e->graphExec);
        e->graphExec = nullptr;
    }
    e->b8 = want;
    return EWG_OK;
}

BiState bicg_template(const ewg_solve_opts* o) {
    BiState b;
    memset(&b, 0, sizeof(b));
    b.relTol = o->linear_solver_tolerance;
    b.absTol = o->linear_solver_abs_tolerance;
    b.maxRes = o->linear_solver_max_error;
    b.maxIter = o->linear_solver_max_iterations;
    b.restartOnBreakdown = o->restart_on_breakdown;
    b.verifyTrue = 0;
    b.w = o->preconditioner_relaxation;
    b.status = ST_PENDING;
    return b;
}

// Preconditioner setup and BiCGStab start for the members of `set` (J, r of their last
// linearization). Members with a singular diagonal block go to `singular` and do not start.
template <typename T>
ewg_status solve_begin(ewg_ensemble* e, const std::vector<int>& set, const ewg_solve_opts* o, std::vector<int>& singular) {
    singular.clear();
    if (set.empty()) return EWG_OK;
    ewg_status s = upload_mask(e, set);
    if (s) return s;
    cudaError_t c;
    if ((c = cudaMemsetAsync(e->flagsF, 0, sizeof(int) * e->M, e->stream)) != cudaSuccess) return ens_fail(e, c, "zero flags");
    Ops<T>::factor(e);
    if ((c = cudaGetLastError()) != cudaSuccess) return ens_fail(e, c, "factor");
    if ((s = sync_read(e, e->hFlagsF, e->flagsF, sizeof(int) * e->M, "read factor flags"))) return s;
    std::vector<int> run;
    for (int m : set) {
        if (e->hFlagsF[m] & 4) singular.push_back(m);
        else run.push_back(m);
    }
    if (run.empty()) return EWG_OK;
    if ((s = upload_mask(e, run))) return s;
    ke_bicg_arm<<<(e->M + 127) / 128, 128, 0, e->stream>>>(e->mask, e->M, bicg_template(o), e->st);
    Ops<T>::rhs_init(e);
    return ens_fail(e, cudaGetLastError(), "bicgstab start");
}

// check_interval BiCGStab iterations of every running member, then the states into hSt
template <typename T>
ewg_status bicg_chunk(ewg_ensemble* e) {
    cudaError_t c;
    if (e->useGraph) {
        ewg_status s = build_graph<T>(e);
        if (s) return s;
        if ((c = cudaGraphLaunch(e->graphExec, e->stream)) != cudaSuccess) return ens_fail(e, c, "graph launch");
    } else {
        for (int k = 0; k < e->checkInterval; ++k) Ops<T>::iteration(e);
        if ((c = cudaGetLastError()) != cudaSuccess) return ens_fail(e, c, "bicgstab launch");
    }
    return sync_read(e, e->hSt, e->st, sizeof(BiState) * e->M, "read state");
}

// BiCGStab to completion on the members of `set` (all other members idle)
template <typename T>
ewg_status solve_set(ewg_ensemble* e, const std::vector<int>& set, const ewg_solve_opts* o, std::vector<int>& singular) {
    ewg_status s;
    cudaError_t c;
    for (int m = 0; m < e->M; ++m) {
        memset(&e->hSt[m], 0, sizeof(BiState));
        e->hSt[m].status = ST_IDLE;
    }
    if ((c = cudaMemcpyAsync(e->st, e->hSt, sizeof(BiState) * e->M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "upload state");
    if ((s = solve_begin<T>(e, set, o, singular))) return s;
    if ((s = set_tiles(e, e->tlB, set))) return s;
    const int maxChunks = o->linear_solver_max_iterations / std::max(1, e->checkInterval) + 4;
    for (int chunk = 0;; ++chunk) {
        if ((s = bicg_chunk<T>(e))) return s;
        bool any = false;
        for (int m : set) any = any || e->hSt[m].status == ST_RUNNING;
        if (!any) break;
        if (chunk > maxChunks) {
            e->err = "ensemble bicgstab: a member never left RUNNING";
            return EWG_ERR_TIMEOUT;
        }
    }
    return EWG_OK;
}

// Per-member state of the time loop: Newton of NewtonMethod::apply (newtonmethod.hh:308-517)
// around each step and the halving retry of FvBaseProblem::timeIntegration (fvbaseproblem.hh:
// 507-550) around the Newton solves.
enum Phase { PH_LIN = 0, PH_SOLVE, PH_DONE, PH_FAILED };

struct MemberRun {
    int phase = PH_LIN;
    int numIt = 0;
    double error = 1e100, lastError = 1e100;
    double dt0 = 0, h = 0;
    int stepsLeft = 0;
    int halvingsStep = 0;  // halvings of the current step
    int lastStatus = EWG_OK;
    // totals over the accepted steps
    int newton = 0, linear = 0, halvings = 0;
};

// All members run `steps` implicit steps. A superstep (1) linearizes the members that need it and
// takes their Newton decisions, (2) starts the BiCGStab solves they need, (3) advances every
// running BiCGStab by check_interval iterations, (4) updates the members whose solve finished. A
// member never waits for another member: whatever phase it is in runs in the next superstep.
template <typename T>
ewg_status ensemble_advance(ewg_ensemble* e, int steps, const double* dt, const ewg_newton_opts* no,
                            const ewg_solve_opts* so, ewg_ensemble_report* rep, ewg_ensemble_stats* stats) {
    const int M = e->M;
    const int maxDiv = e->maxDiv;
    if (ewg_status o = ens_set_order(e, so)) return o;
    std::vector<MemberRun> mr(M);
    for (int m = 0; m < M; ++m) {
        if (!(dt[m] > 0)) { e->err = "dt must be positive"; return EWG_ERR_INVALID; }
        mr[m].dt0 = mr[m].h = dt[m];
        mr[m].stepsLeft = steps;
    }
    ewg_ensemble_stats S;
    memset(&S, 0, sizeof(S));
    ewg_status s;
    cudaError_t c;
    float ms = 0;
    auto converged = [&](const MemberRun& n) { return n.error <= no->newton_tolerance; };
    auto proceed = [&](const MemberRun& n) {
        if (n.numIt < 1) return true;
        if (converged(n)) return false;
        if (n.numIt >= no->newton_max_iterations) return n.error * 4.0 < n.lastError;
        return true;
    };
    // the BiCGStab state of every member starts idle
    for (int m = 0; m < M; ++m) {
        memset(&e->hSt[m], 0, sizeof(BiState));
        e->hSt[m].status = ST_IDLE;
    }
    if ((c = cudaMemcpyAsync(e->st, e->hSt, sizeof(BiState) * M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "upload state");
    std::vector<int> accepted, failed;
    auto fail = [&](int m, int status) {
        mr[m].lastStatus = status;
        failed.push_back(m);
    };
    auto accept = [&](int m) { accepted.push_back(m); };
    // restore failed members, advance accepted ones, and set up their next attempt / step
    auto settle = [&]() -> ewg_status {
        ewg_status q;
        if ((q = levels(e, failed, 2))) return q;
        if ((q = levels(e, accepted, 1))) return q;
        for (int m : failed) {
            MemberRun& n = mr[m];
            n.halvingsStep += 1;
            if (n.halvingsStep >= maxDiv) { n.phase = PH_FAILED; continue; }
            n.h *= 0.5;
            n.numIt = 0;
            n.error = n.lastError = 1e100;
            n.phase = PH_LIN;
        }
        for (int m : accepted) {
            MemberRun& n = mr[m];
            n.newton += n.numIt;
            n.halvings += n.halvingsStep;
            n.lastStatus = EWG_OK;
            if (--n.stepsLeft == 0) { n.phase = PH_DONE; continue; }
            n.h = n.dt0;
            n.halvingsStep = 0;
            n.numIt = 0;
            n.error = n.lastError = 1e100;
            n.phase = PH_LIN;
        }
        failed.clear();
        accepted.clear();
        return EWG_OK;
    };
    const int maxSupersteps = 10000000;
    for (int ss = 0; ss < maxSupersteps; ++ss) {
        S.supersteps += 1;
        // ---- (1) linearization and the Newton decisions that follow it
        std::vector<int> lin;
        for (int m = 0; m < M; ++m)
            if (mr[m].phase == PH_LIN) {
                mr[m].lastError = mr[m].error;
                e->hDt[m] = mr[m].h;
                lin.push_back(m);
            }
        std::vector<int> newSolve;
        if (!lin.empty()) {
            S.rounds += 1;
            cudaEventRecord(e->ev0, e->stream);
            if ((s = linearize_set<T>(e, lin, true))) return s;
            cudaEventRecord(e->ev1, e->stream);
            cudaEventSynchronize(e->ev1);
            cudaEventElapsedTime(&ms, e->ev0, e->ev1);
            S.t_linearize += ms * 1e-3;
            for (int m : lin) {
                MemberRun& n = mr[m];
                if (e->hFlags[m] & 1) { fail(m, EWG_ERR_NONFINITE); continue; }
                n.lastError = n.error;
                n.error = err_of(e, m);
                if (n.error > no->newton_max_error) { fail(m, EWG_ERR_MAX_ERROR); continue; }
                if (!proceed(n)) {
                    ++n.numIt;
                    if (converged(n)) accept(m);
                    else fail(m, EWG_ERR_NOT_CONVERGED);
                    continue;
                }
                newSolve.push_back(m);
            }
        }
        // ---- (2) solves of the members that need a Newton correction
        if (!newSolve.empty()) {
            std::vector<int> singular;
            cudaEventRecord(e->ev0, e->stream);
            if ((s = solve_begin<T>(e, newSolve, so, singular))) return s;
            cudaEventRecord(e->ev1, e->stream);
            cudaEventSynchronize(e->ev1);
            cudaEventElapsedTime(&ms, e->ev0, e->ev1);
            S.t_solve += ms * 1e-3;
            for (int m : singular) fail(m, EWG_ERR_BREAKDOWN);
            for (int m : newSolve)
                if (std::find(singular.begin(), singular.end(), m) == singular.end()) mr[m].phase = PH_SOLVE;
        }
        if ((s = settle())) return s;
        // ---- (3) every running BiCGStab advances
        std::vector<int> solving;
        for (int m = 0; m < M; ++m)
            if (mr[m].phase == PH_SOLVE) solving.push_back(m);
        if (!solving.empty()) {
            cudaEventRecord(e->ev0, e->stream);
            if ((s = set_tiles(e, e->tlB, solving))) return s;
            if ((s = bicg_chunk<T>(e))) return s;
            cudaEventRecord(e->ev1, e->stream);
            cudaEventSynchronize(e->ev1);
            cudaEventElapsedTime(&ms, e->ev0, e->ev1);
            S.t_solve += ms * 1e-3;
            // ---- (4) Newton update of the members whose solve ended
            std::vector<int> upd;
            for (int m : solving) {
                const BiState& b = e->hSt[m];
                if (b.status == ST_RUNNING) {
                    if (b.iter > so->linear_solver_max_iterations + 8) {
                        e->err = "ensemble bicgstab: a member never left RUNNING";
                        return EWG_ERR_TIMEOUT;
                    }
                    continue;
                }
                mr[m].linear += b.iter;
                S.linear_iterations += b.iter;
                S.cell_iterations += (double)e->hm[m].P.N * b.iter;
                if (b.status == ST_CONVERGED) upd.push_back(m);
                else fail(m, b.status == ST_BREAKDOWN ? EWG_ERR_BREAKDOWN : EWG_ERR_NOT_CONVERGED);
                mr[m].phase = PH_LIN;  // provisional; settle() or the checks below decide
            }
            if (!upd.empty()) {
                cudaEventRecord(e->ev0, e->stream);
                if ((s = upload_mask(e, upd))) return s;
                if ((c = cudaMemsetAsync(e->flagsU, 0, sizeof(int) * M, e->stream)) != cudaSuccess) return ens_fail(e, c, "zero flags");
                Ops<T>::update(e);
                if ((c = cudaGetLastError()) != cudaSuccess) return ens_fail(e, c, "update");
                if ((s = sync_read(e, e->hFlagsU, e->flagsU, sizeof(int) * M, "read update flags"))) return s;
                cudaEventRecord(e->ev1, e->stream);
                cudaEventSynchronize(e->ev1);
                cudaEventElapsedTime(&ms, e->ev0, e->ev1);
                S.t_update += ms * 1e-3;
                for (int m : upd) {
                    MemberRun& n = mr[m];
                    if (e->hFlagsU[m] & 2) { fail(m, EWG_ERR_NONFINITE); continue; }
                    ++n.numIt;
                    // the loop-top test of NewtonMethod::apply (while (proceed_()))
                    if (!proceed(n)) {
                        if (converged(n)) accept(m);
                        else fail(m, EWG_ERR_NOT_CONVERGED);
                    }
                }
            }
            if ((s = settle())) return s;
        }
        bool active = false;
        for (int m = 0; m < M; ++m) active = active || mr[m].phase == PH_LIN || mr[m].phase == PH_SOLVE;
        if (!active) break;
    }
    if ((s = ens_fail(e, cudaStreamSynchronize(e->stream), "sync advance"))) return s;
    bool allOk = true;
    for (int m = 0; m < M; ++m) {
        const MemberRun& n = mr[m];
        if (rep) {
            rep[m].status = n.phase == PH_DONE ? EWG_OK : n.lastStatus;
            rep[m].newton_iterations = n.phase == PH_DONE ? n.newton : n.numIt;
            rep[m].linear_iterations = n.linear;
            rep[m].halvings = n.halvings + (n.phase == PH_DONE ? 0 : n.halvingsStep);
            rep[m].dt = n.h;
            rep[m].error = n.error;
        }
        allOk = allOk && n.phase == PH_DONE;
    }
    if (stats) *stats = S;
    if (!allOk) {
        e->err = "a member's time step failed after the allowed halvings";
        return EWG_ERR_NOT_CONVERGED;
    }
    return EWG_OK;
}

// ---- Newton decisions on the device ---------------------------------------------------------------
//
// ensemble_advance_device runs the supersteps of ensemble_advance with every per-member decision
// taken on the device by single-block scheduling kernels (kd_*), and captures one whole superstep as
// the body of a CUDA graph WHILE node: one graph launch runs supersteps until no member is active,
// without returning to the host. The work kernels, their order and the member set of every launch
// are those of ensemble_advance (the tile lists are compacted on the device in member order, as
// set_tiles does on the host), so both advance the members to the same bits.

__device__ __forceinline__ bool d_converged(const RunD& n, const NewtonD& no) { return n.error <= no.tol; }
// NewtonMethod::proceed_ (newtonmethod.hh:620-636), as ensemble_advance's proceed
__device__ __forceinline__ bool d_proceed(const RunD& n, const NewtonD& no) {
    if (n.numIt < 1) return true;
    if (d_converged(n, no)) return false;
    if (n.numIt >= no.maxIt) return n.error * 4.0 < n.lastError;
    return true;
}
__device__ __forceinline__ void d_fail(RunD& n, int status) {
    n.lastStatus = status;
    n.fail = 1;
}

// tile list of the members with sel[m] != 0, in member order (set_tiles); one block
__global__ void kd_tiles(const EnsMember* __restrict__ mem, const int2* __restrict__ allTiles, int M,
                         const int* __restrict__ sel, int* __restrict__ prefix, int2* __restrict__ out,
                         int* __restrict__ outN) {
    if (threadIdx.x == 0) {
        int n = 0;
        for (int m = 0; m < M; ++m) {
            prefix[m] = n;
            if (sel[m]) n += mem[m].ntiles;
        }
        *outN = n;
    }
    __syncthreads();
    for (int m = 0; m < M; ++m) {
        if (!sel[m]) continue;
        const int t0 = mem[m].tile0, nt = mem[m].ntiles, o = prefix[m];
        for (int k = threadIdx.x; k < nt; k += blockDim.x) out[o + k] = allTiles[t0 + k];
    }
}

// (1) the members that linearize: mask, their step sizes, cleared error maxima and flags
__global__ void kd_lin_begin(RunD* __restrict__ run, int M, int* __restrict__ mask, double* __restrict__ dtArr,
                             unsigned long long* __restrict__ errmax, int* __restrict__ flags, SchedD* __restrict__ sch) {
    int any = 0;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        RunD& n = run[m];
        const int sel = n.phase == PH_LIN;
        if (sel) {
            n.lastError = n.error;
            dtArr[m] = n.h;
        }
        mask[m] = sel;
        errmax[m] = 0ull;
        flags[m] = 0;
        any |= sel;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0 && any) sch->rounds += 1;
}

// (1) Newton decisions after the linearization; mask becomes the members that need a correction
__global__ void kd_lin_decide(RunD* __restrict__ run, int M, int* __restrict__ mask,
                              const unsigned long long* __restrict__ errmax, const int* __restrict__ flags,
                              int* __restrict__ flagsF, NewtonD no) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        flagsF[m] = 0;
        if (!mask[m]) continue;
        RunD& n = run[m];
        int solve = 0;
        if (flags[m] & 1) {
            d_fail(n, EWG_ERR_NONFINITE);
        } else {
            n.lastError = n.error;
            n.error = __longlong_as_double((long long)errmax[m]);
            if (n.error > no.maxError) {
                d_fail(n, EWG_ERR_MAX_ERROR);
            } else if (!d_proceed(n, no)) {
                ++n.numIt;
                if (d_converged(n, no)) n.accept = 1;
                else d_fail(n, EWG_ERR_NOT_CONVERGED);
            } else {
                solve = 1;
            }
        }
        mask[m] = solve;
    }
}

// (2) after the preconditioner setup: a singular diagonal block fails the member, the others solve
__global__ void kd_factor_decide(RunD* __restrict__ run, int M, int* __restrict__ mask, const int* __restrict__ flagsF) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        if (!mask[m]) continue;
        if (flagsF[m] & 4) {
            d_fail(run[m], EWG_ERR_BREAKDOWN);
            mask[m] = 0;
        } else {
            run[m].phase = PH_SOLVE;
        }
    }
}

// settle, part 1: the failed and the accepted members as masks (their levels are reset / advanced)
__global__ void kd_settle_masks(const RunD* __restrict__ run, int M, int* __restrict__ maskF, int* __restrict__ maskA) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        maskF[m] = run[m].fail;
        maskA[m] = run[m].accept;
    }
}

// settle, part 2: retry with half the step, or the next step (ensemble_advance's settle)
__global__ void kd_settle(RunD* __restrict__ run, int M, int maxDiv) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        RunD& n = run[m];
        if (n.fail) {
            n.fail = 0;
            n.halvingsStep += 1;
            if (n.halvingsStep >= maxDiv) {
                n.phase = PH_FAILED;
            } else {
                n.h *= 0.5;
                n.numIt = 0;
                n.error = n.lastError = 1e100;
                n.phase = PH_LIN;
            }
        }
        if (n.accept) {
            n.accept = 0;
            n.newton += n.numIt;
            n.halvings += n.halvingsStep;
            n.lastStatus = EWG_OK;
            if (--n.stepsLeft == 0) {
                n.phase = PH_DONE;
            } else {
                n.h = n.dt0;
                n.halvingsStep = 0;
                n.numIt = 0;
                n.error = n.lastError = 1e100;
                n.phase = PH_LIN;
            }
        }
    }
}

// (3) the members whose BiCGStab runs this superstep
__global__ void kd_solve_select(const RunD* __restrict__ run, int M, int* __restrict__ maskS) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) maskS[m] = run[m].phase == PH_SOLVE;
}

// (4) after the BiCGStab iterations: members whose solve ended take the Newton update (mask) or fail
__global__ void kd_solve_decide(RunD* __restrict__ run, int M, const int* __restrict__ maskS,
                                const BiState* __restrict__ st, const EnsMember* __restrict__ mem, int* __restrict__ mask,
                                int* __restrict__ flagsU, int maxIter, SchedD* __restrict__ sch) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        flagsU[m] = 0;
        int upd = 0;
        if (maskS[m]) {
            const BiState& b = st[m];
            if (b.status == ST_RUNNING) {
                if (b.iter > maxIter + 8) atomicExch(&sch->error, (int)EWG_ERR_TIMEOUT);
            } else {
                RunD& n = run[m];
                n.linear += b.iter;
                atomicAdd(&sch->linearIterations, b.iter);
                atomicAdd(&sch->cellIterations, (double)mem[m].P.N * b.iter);
                if (b.status == ST_CONVERGED) upd = 1;
                else d_fail(n, b.status == ST_BREAKDOWN ? EWG_ERR_BREAKDOWN : EWG_ERR_NOT_CONVERGED);
                n.phase = PH_LIN;  // provisional; settle or the update decision decides
            }
        }
        mask[m] = upd;
    }
}

// (4) after the Newton update: the loop-top test of NewtonMethod::apply (while (proceed_()))
__global__ void kd_update_decide(RunD* __restrict__ run, int M, const int* __restrict__ mask,
                                 const int* __restrict__ flagsU, NewtonD no) {
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        if (!mask[m]) continue;
        RunD& n = run[m];
        if (flagsU[m] & 2) {
            d_fail(n, EWG_ERR_NONFINITE);
            continue;
        }
        ++n.numIt;
        if (!d_proceed(n, no)) {
            if (d_converged(n, no)) n.accept = 1;
            else d_fail(n, EWG_ERR_NOT_CONVERGED);
        }
    }
}

// end of a superstep: another one while a member is active, no member timed out and the launch's
// superstep bound is not reached
__global__ void kd_superstep_end(const RunD* __restrict__ run, int M, SchedD* __restrict__ sch,
                                 cudaGraphConditionalHandle loop) {
    int act = 0;
    for (int m = threadIdx.x; m < M; m += blockDim.x) act |= run[m].phase == PH_LIN || run[m].phase == PH_SOLVE;
    act = __syncthreads_or(act);
    if (threadIdx.x == 0) {
        sch->active = act;
        sch->supersteps += 1;
        const bool more = act && sch->error == 0 && sch->supersteps < sch->limit;
        cudaGraphSetConditional(loop, more ? 1u : 0u);
    }
}

// supersteps per graph launch: the host reads the scheduler state between launches
constexpr long long kSuperstepsPerLaunch = 4096;

ewg_status ensure_sched(ewg_ensemble* e) {
    if (e->dRun) return EWG_OK;
    const int M = e->M;
    cudaError_t c = cudaMalloc(&e->dRun, sizeof(RunD) * M);
    if (c == cudaSuccess) c = cudaMalloc(&e->dSched, sizeof(SchedD));
    if (c == cudaSuccess) c = cudaMalloc(&e->dPrefix, sizeof(int) * M);
    if (c == cudaSuccess) c = cudaMalloc(&e->maskF, sizeof(int) * M);
    if (c == cudaSuccess) c = cudaMalloc(&e->maskA, sizeof(int) * M);
    if (c == cudaSuccess) c = cudaMalloc(&e->maskS, sizeof(int) * M);
    if (c == cudaSuccess) c = cudaMalloc(&e->dTilesAll, sizeof(int2) * std::max(1, e->nTiles));
    if (c == cudaSuccess) c = cudaMallocHost(&e->hRun, sizeof(RunD) * M);
    if (c == cudaSuccess) c = cudaMallocHost(&e->hSched, sizeof(SchedD));
    if (c == cudaSuccess && e->nTiles > 0)
        c = cudaMemcpyAsync(e->dTilesAll, e->hTiles.data(), sizeof(int2) * e->nTiles, cudaMemcpyHostToDevice, e->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
    return ens_fail(e, c, "allocate device scheduler");
}

void kd_tile_list(ewg_ensemble* e, const int* sel, ewg_ensemble::TileList& tl) {
    kd_tiles<<<1, 256, 0, e->stream>>>(e->dm, e->dTilesAll, e->M, sel, e->dPrefix, tl.d, tl.dn);
}

// settle on the device: levels of the failed (x0 = x1) and accepted (x1 = x0) members, then their
// next attempt or step
void kd_settle_all(ewg_ensemble* e) {
    cudaStream_t s = e->stream;
    kd_settle_masks<<<1, 256, 0, s>>>(e->dRun, e->M, e->maskF, e->maskA);
    kd_tile_list(e, e->maskF, e->tlA);
    ke_levels<<<e->grid[EC_CELL], kEnsTile, 0, s>>>(e->dm, e->tlA.d, e->tlA.dn, e->maskF, 2, e->x0, e->x1, e->sold);
    kd_tile_list(e, e->maskA, e->tlA);
    ke_levels<<<e->grid[EC_CELL], kEnsTile, 0, s>>>(e->dm, e->tlA.d, e->tlA.dn, e->maskA, 1, e->x0, e->x1, e->sold);
    kd_settle<<<1, 256, 0, s>>>(e->dRun, e->M, e->maxDiv);
}

// one superstep of ensemble_advance, every launch on the ensemble stream (captured into the body)
template <typename T>
void superstep_device(ewg_ensemble* e, const NewtonD& nd, const ewg_solve_opts* so, cudaGraphConditionalHandle loop) {
    cudaStream_t s = e->stream;
    const int M = e->M;
    // (1) linearization and the Newton decisions that follow it
    kd_lin_begin<<<1, 256, 0, s>>>(e->dRun, M, e->mask, e->dtArr, e->errmax, e->flags, e->dSched);
    kd_tile_list(e, e->mask, e->tlA);
    Ops<T>::intensive(e);
    Ops<T>::assemble(e, true);
    kd_lin_decide<<<1, 256, 0, s>>>(e->dRun, M, e->mask, e->errmax, e->flags, e->flagsF, nd);
    // (2) preconditioner setup and BiCGStab start of the members that need a correction
    kd_tile_list(e, e->mask, e->tlA);
    Ops<T>::factor(e);
    kd_factor_decide<<<1, 256, 0, s>>>(e->dRun, M, e->mask, e->flagsF);
    kd_tile_list(e, e->mask, e->tlA);
    ke_bicg_arm<<<(M + 127) / 128, 128, 0, s>>>(e->mask, M, bicg_template(so), e->st);
    Ops<T>::rhs_init(e);
    kd_settle_all(e);
    // (3) every running BiCGStab advances by check_interval iterations
    kd_solve_select<<<1, 256, 0, s>>>(e->dRun, M, e->maskS);
    kd_tile_list(e, e->maskS, e->tlB);
    for (int k = 0; k < e->checkInterval; ++k) Ops<T>::iteration(e);
    // (4) Newton update of the members whose solve ended
    kd_solve_decide<<<1, 256, 0, s>>>(e->dRun, M, e->maskS, e->st, e->dm, e->mask, e->flagsU,
                                      so->linear_solver_max_iterations, e->dSched);
    kd_tile_list(e, e->mask, e->tlA);
    Ops<T>::update(e);
    kd_update_decide<<<1, 256, 0, s>>>(e->dRun, M, e->mask, e->flagsU, nd);
    kd_settle_all(e);
    kd_superstep_end<<<1, 256, 0, s>>>(e->dRun, M, e->dSched, loop);
}

// graph: one WHILE node whose body is a superstep
template <typename T>
ewg_status build_device_advance(ewg_ensemble* e, const NewtonD& nd, const ewg_solve_opts* so, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    cudaError_t c = cudaGraphCreate(&g, 0);
    if (c != cudaSuccess) return ens_fail(e, c, "create graph");
    cudaGraphConditionalHandle loop = 0;
    c = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (c == cudaSuccess) c = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    if (c == cudaSuccess)
        c = cudaStreamBeginCaptureToGraph(e->stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (c == cudaSuccess) {
        superstep_device<T>(e, nd, so, loop);
        cudaGraph_t body = nullptr;
        const cudaError_t launch = cudaGetLastError();
        c = cudaStreamEndCapture(e->stream, &body);
        if (c == cudaSuccess) c = launch;
    }
    if (c == cudaSuccess) c = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return ens_fail(e, c, "device advance graph");
}

// ensemble_advance with the decisions on the device: the host starts the graph, reads the
// scheduler state between launches (every kSuperstepsPerLaunch supersteps) and the members' runs at
// the end. Stats: t_solve is the device time of the whole advance (phases are not timed apart).
template <typename T>
ewg_status ensemble_advance_device(ewg_ensemble* e, int steps, const double* dt, const ewg_newton_opts* no,
                                   const ewg_solve_opts* so, ewg_ensemble_report* rep, ewg_ensemble_stats* stats) {
    const int M = e->M;
    for (int m = 0; m < M; ++m)
        if (!(dt[m] > 0)) { e->err = "dt must be positive"; return EWG_ERR_INVALID; }
    if (ewg_status o = ens_set_order(e, so)) return o;
    ewg_status s = ensure_sched(e);
    if (s) return s;
    cudaError_t c;
    for (int m = 0; m < M; ++m) {
        RunD& n = e->hRun[m];
        memset(&n, 0, sizeof(n));
        n.phase = PH_LIN;
        n.error = n.lastError = 1e100;
        n.dt0 = n.h = dt[m];
        n.stepsLeft = steps;
        n.lastStatus = EWG_OK;
        memset(&e->hSt[m], 0, sizeof(BiState));
        e->hSt[m].status = ST_IDLE;
    }
    memset(e->hSched, 0, sizeof(SchedD));
    e->hSched->limit = kSuperstepsPerLaunch;
    if ((c = cudaMemcpyAsync(e->st, e->hSt, sizeof(BiState) * M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess ||
        (c = cudaMemcpyAsync(e->dRun, e->hRun, sizeof(RunD) * M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess ||
        (c = cudaMemcpyAsync(e->dSched, e->hSched, sizeof(SchedD), cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "upload scheduler state");
    const NewtonD nd{no->newton_tolerance, no->newton_max_error, no->newton_max_iterations};
    cudaGraphExec_t exec = nullptr;
    if ((s = build_device_advance<T>(e, nd, so, &exec))) return s;
    auto done = [&](ewg_status r) {
        cudaGraphExecDestroy(exec);
        return r;
    };
    cudaEventRecord(e->ev0, e->stream);
    const long long maxSupersteps = 10000000;
    for (;;) {
        if ((c = cudaGraphLaunch(exec, e->stream)) != cudaSuccess) return done(ens_fail(e, c, "graph launch"));
        if ((s = sync_read(e, e->hSched, e->dSched, sizeof(SchedD), "read scheduler state"))) return done(s);
        if (e->hSched->error) {
            e->err = "ensemble bicgstab: a member never left RUNNING";
            return done((ewg_status)e->hSched->error);
        }
        if (!e->hSched->active) break;
        if (e->hSched->supersteps >= maxSupersteps) {
            e->err = "ensemble advance: superstep limit reached";
            return done(EWG_ERR_TIMEOUT);
        }
        e->hSched->limit = e->hSched->supersteps + kSuperstepsPerLaunch;
        if ((c = cudaMemcpyAsync(&e->dSched->limit, &e->hSched->limit, sizeof(long long), cudaMemcpyHostToDevice,
                                 e->stream)) != cudaSuccess)
            return done(ens_fail(e, c, "upload superstep bound"));
    }
    cudaEventRecord(e->ev1, e->stream);
    if ((s = sync_read(e, e->hRun, e->dRun, sizeof(RunD) * M, "read member runs"))) return done(s);
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    bool allOk = true;
    for (int m = 0; m < M; ++m) {
        const RunD& n = e->hRun[m];
        if (rep) {
            rep[m].status = n.phase == PH_DONE ? EWG_OK : n.lastStatus;
            rep[m].newton_iterations = n.phase == PH_DONE ? n.newton : n.numIt;
            rep[m].linear_iterations = n.linear;
            rep[m].halvings = n.halvings + (n.phase == PH_DONE ? 0 : n.halvingsStep);
            rep[m].dt = n.h;
            rep[m].error = n.error;
        }
        allOk = allOk && n.phase == PH_DONE;
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->rounds = e->hSched->rounds;
        stats->linear_iterations = e->hSched->linearIterations;
        stats->cell_iterations = e->hSched->cellIterations;
        stats->t_solve = ms * 1e-3;
        stats->supersteps = (int32_t)e->hSched->supersteps;
    }
    if (!allOk) {
        e->err = "a member's time step failed after the allowed halvings";
        return done(EWG_ERR_NOT_CONVERGED);
    }
    return done(EWG_OK);
}

// Time every launch shape of each kernel class on the current state and keep the fastest.
template <typename T>
ewg_status autotune(ewg_ensemble* e, const double* dt, const ewg_solve_opts* so) {
    if (ewg_status o = ens_set_order(e, so)) return o;
    std::vector<int> all(e->M);
    for (int m = 0; m < e->M; ++m) {
        all[m] = m;
        e->hDt[m] = dt[m];
    }
    const int mults[] = {1, 2, 3, 4, 6, 8};
    ewg_status s;
    cudaError_t c;
    auto timeit = [&](auto&& launch, int reps) -> double {
        double best = 1e30;
        for (int r = 0; r < reps; ++r) {
            cudaEventRecord(e->tev[0], e->stream);
            launch();
            cudaEventRecord(e->tev[1], e->stream);
            cudaEventSynchronize(e->tev[1]);
            float ms = 0;
            cudaEventElapsedTime(&ms, e->tev[0], e->tev[1]);
            best = std::min(best, (double)ms);
        }
        return best;
    };
    if ((s = upload_mask(e, all))) return s;
    if ((c = cudaMemcpyAsync(e->dtArr, e->hDt, sizeof(double) * e->M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "upload dt");
    // linearization kernels are idempotent in x0: time them directly
    for (int cls : {EC_INTENSIVE, EC_ASSEMBLE}) {
        const int base = e->grid[cls];
        int bestG = base, bestV = e->asmVariant;
        double best = 1e30;
        const int variants[] = {3, 2};
        for (int vi = 0; vi < (cls == EC_ASSEMBLE ? 2 : 1); ++vi) {
            if (cls == EC_ASSEMBLE) e->asmVariant = variants[vi];
            for (int mu : mults) {
                e->grid[cls] = std::min(e->nTiles, e->numSMs * mu);
                const double t = timeit([&] { cls == EC_INTENSIVE ? Ops<T>::intensive(e) : Ops<T>::assemble(e, true); }, 3);
                if (t < best) { best = t; bestG = e->grid[cls]; bestV = e->asmVariant; }
            }
        }
        e->grid[cls] = bestG;
        if (cls == EC_ASSEMBLE) e->asmVariant = bestV;
    }
    if ((c = cudaGetLastError()) != cudaSuccess) return ens_fail(e, c, "tune linearize");
    // a real preconditioner and BiCGStab start; each timed launch starts from the saved state
    if ((s = linearize_set<T>(e, all, true))) return s;
    std::vector<int> singular;
    ewg_solve_opts o = *so;
    o.linear_solver_max_iterations = 1;  // one chunk is enough to set up; the state is reset below
    const bool g = e->useGraph;
    e->useGraph = false;
    s = solve_set<T>(e, all, &o, singular);
    e->useGraph = g;
    if (s) return s;
    // restart every member from its initial BiCGStab state
    if ((s = upload_mask(e, all))) return s;
    for (int m = 0; m < e->M; ++m) e->hSt[m].status = ST_PENDING;
    if ((c = cudaMemcpyAsync(e->st, e->hSt, sizeof(BiState) * e->M, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "upload state");
    Ops<T>::rhs_init(e);
    if ((c = cudaMemcpyAsync(e->stSave, e->st, sizeof(BiState) * e->M, cudaMemcpyDeviceToDevice, e->stream)) != cudaSuccess)
        return ens_fail(e, c, "save state");
    if ((s = set_tiles(e, e->tlB, all))) return s;
    for (int cls : {EC_P, EC_ILU_BLACK, EC_ILU_RED, EC_SPMV_ALPHA, EC_HS, EC_SPMV_OMEGA, EC_XR}) {
        int bestG = e->grid[cls];
        double best = 1e30;
        for (int mu : mults) {
            e->grid[cls] = std::min(e->nTiles, e->numSMs * mu);
            const double t = timeit([&] {
                cudaMemcpyAsync(e->st, e->stSave, sizeof(BiState) * e->M, cudaMemcpyDeviceToDevice, e->stream);
                Ops<T>::kernel(e, cls, 0);
            }, 3);
            if (t < best) { best = t; bestG = e->grid[cls]; }
        }
        e->grid[cls] = bestG;
    }
    if ((c = cudaGetLastError()) != cudaSuccess) return ens_fail(e, c, "tune bicgstab");
    e->grid[EC_CELL] = e->grid[EC_P];
    e->grid[EC_FACTOR] = e->grid[EC_ILU_BLACK];
    if (e->graphExec) {
        cudaGraphExecDestroy(e->graphExec);
        e->graphExec = nullptr;
    }
    e->tuned = true;
    return ens_fail(e, cudaStreamSynchronize(e->stream), "sync tune");
}

ewg_status check_ens(ewg_ensemble* e) { return e ? EWG_OK : EWG_ERR_INVALID; }

}  // namespace

extern "C" {

const char* ewg_ensemble_create_error(void) { return g_ensCreateError.c_str(); }
const char* ewg_ensemble_last_error(const ewg_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

void ewg_default_ensemble_opts(ewg_ensemble_opts* o) {
    if (!o) return;
    o->precision = EWG_PRECISION_MIXED;
    o->use_graph = 1;
    o->check_interval = 8;
    o->max_divisions = 10;
}

void ewg_ensemble_destroy(ewg_ensemble* e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->graphExec) cudaGraphExecDestroy(e->graphExec);
    void* ps[] = {e->dm, e->x0, e->x1, e->sold, e->r, e->stage, e->perm, e->lens, e->iq, e->geo, e->J,
                  e->Dinv, e->L, e->kx, e->kr, e->kr0, e->kv, e->kp, e->ky, e->kz, e->kb, e->partials, e->counters,
                  e->st, e->stSave, e->mask, e->errmax, e->flags, e->flagsF, e->flagsU, e->dtArr,
                  e->dRun, e->dSched, e->dPrefix, e->dTilesAll, e->maskF, e->maskA, e->maskS,
                  e->A8, e->L8, e->Dinv8, e->E8, e->W8};
    for (void* p : ps)
        if (p) cudaFree(p);
    void* hs[] = {e->hSt, e->hMask, e->hErr, e->hFlags, e->hFlagsF, e->hFlagsU, e->hDt, e->hRun, e->hSched};
    for (void* p : hs)
        if (p) cudaFreeHost(p);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    for (cudaEvent_t ev : e->tev)
        if (ev) cudaEventDestroy(ev);
    if (e->maskEv) cudaEventDestroy(e->maskEv);
    for (ewg_ensemble::TileList* tl : {&e->tlA, &e->tlB}) {
        if (tl->d) cudaFree(tl->d);
        if (tl->dn) cudaFree(tl->dn);
        if (tl->h) cudaFreeHost(tl->h);
        if (tl->hn) cudaFreeHost(tl->hn);
        if (tl->ev) cudaEventDestroy(tl->ev);
    }
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

ewg_status ewg_ensemble_create(int32_t members, const ewg_grid* grids, const ewg_problem* problems,
                               const double* const* perms, const ewg_ensemble_opts* opts, ewg_ensemble** out) {
    g_ensCreateError.clear();
    if (!out || !grids || !problems || !perms || members < 1) {
        g_ensCreateError = "null argument or no members";
        return EWG_ERR_INVALID;
    }
    *out = nullptr;
    ewg_ensemble_opts dflt;
    ewg_default_ensemble_opts(&dflt);
    if (!opts) opts = &dflt;
    if (opts->precision != EWG_PRECISION_FP64 && opts->precision != EWG_PRECISION_MIXED) {
        g_ensCreateError = "precision must be EWG_PRECISION_FP64 or EWG_PRECISION_MIXED";
        return EWG_ERR_INVALID;
    }
    int64_t total = 0;
    int64_t tiles = 0;
    for (int m = 0; m < members; ++m) {
        const ewg_grid& g = grids[m];
        if (g.dim != 3 || g.nx < 2 || (g.nx & 1) || g.ny < 1 || g.nz < 1 || g.k_origin != 0 || !perms[m]) {
            g_ensCreateError = "member " + std::to_string(m) + ": ensembles take whole 3D grids (k_origin 0) with even nx >= 2 and a permeability field";
            return EWG_ERR_INVALID;
        }
        const int64_t n = (int64_t)g.nx * g.ny * g.nz;
        total += n;
        tiles += (n / 2 + kEnsTileH - 1) / kEnsTileH;
    }
    if (total >= ((int64_t)1 << 31) || tiles >= ((int64_t)1 << 31)) {
        g_ensCreateError = "ensemble too large (2^31 cells)";
        return EWG_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        g_ensCreateError = "no CUDA device";
        return EWG_ERR_NO_DEVICE;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10) {
        g_ensCreateError = "device is not sm_100 (B200)";
        return EWG_ERR_NO_DEVICE;
    }
    ewg_ensemble* e = new ewg_ensemble();
    e->M = members;
    e->device = dev;
    e->numSMs = prop.multiProcessorCount;
    e->precision = opts->precision;
    e->useGraph = opts->use_graph != 0;
    e->checkInterval = opts->check_interval > 0 ? opts->check_interval : 8;
    e->maxDiv = opts->max_divisions > 0 ? opts->max_divisions : 10;
    e->total = total;
    cudaError_t c = cudaSuccess;
    auto failc = [&](const char* what) {
        g_ensCreateError = std::string(what) + ": " + cudaGetErrorString(c);
        ewg_ensemble_destroy(e);
        return EWG_ERR_CUDA;
    };
    if ((c = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) return failc("stream");
    cudaEvent_t* evs[] = {&e->ev0, &e->ev1, &e->tev[0], &e->tev[1], &e->maskEv};
    for (cudaEvent_t* ev : evs)
        if ((c = cudaEventCreate(ev)) != cudaSuccess) return failc("event");
    // members, tiles, geometry
    std::vector<FaceGeo> geoAll;
    e->hm.resize(members);
    int64_t off = 0;
    for (int m = 0; m < members; ++m) {
        EnsMember& em = e->hm[m];
        memset(&em, 0, sizeof(em));
        build_phys(em.P, &grids[m], &problems[m]);
        if ((c = boundary_constants(em.P, e->stream)) != cudaSuccess) return failc("boundary constants");
        em.off = off;
        em.geoOff = (int64_t)geoAll.size();
        std::vector<FaceGeo> g;
        build_face_geo(em.P, g);
        geoAll.insert(geoAll.end(), g.begin(), g.end());
        em.tile0 = (int32_t)e->hTiles.size();
        const int64_t nt = (em.P.Nh + kEnsTileH - 1) / kEnsTileH;
        em.ntiles = (int32_t)nt;
        for (int64_t t = 0; t < nt; ++t) e->hTiles.push_back(make_int2(m, (int)(t * kEnsTileH)));
        off += em.P.N;
    }
    e->nTiles = (int)e->hTiles.size();
    e->b8ok = true;
    for (int m = 0; m < members; ++m) e->b8ok = e->b8ok && e->hm[m].P.b8ok;
    const bool mixed = e->precision == EWG_PRECISION_MIXED;
    const size_t sT = mixed ? sizeof(float) : sizeof(double);
    const size_t sV = 2 * sT;
    struct A { void** p; size_t bytes; const char* what; };
    const A allocs[] = {
        {(void**)&e->dm, sizeof(EnsMember) * members, "members"},
        {(void**)&e->x0, sizeof(double2) * total, "x0"},
        {(void**)&e->x1, sizeof(double2) * total, "x1"},
        {(void**)&e->sold, sizeof(double2) * total, "storage"},
        {(void**)&e->r, sizeof(double2) * total, "residual"},
        {(void**)&e->stage, sizeof(double2) * total, "staging"},
        {(void**)&e->perm, sizeof(double) * total, "perm"},
        {(void**)&e->lens, (size_t)total, "lens"},
        {(void**)&e->iq, sizeof(double) * 6 * total, "intensive cache"},
        {(void**)&e->geo, sizeof(FaceGeo) * geoAll.size(), "geometry"},
        {&e->J, sT * kEnsBands * 4 * total, "jacobian"},
        {&e->Dinv, sT * 4 * total, "dinv"},
        {&e->L, sT * 12 * total, "ilu L"},
        {&e->kx, sV * total, "x"}, {&e->kr, sV * total, "r"}, {&e->kr0, sV * total, "r0"}, {&e->kv, sV * total, "v"},
        {&e->kp, sV * total, "p"}, {&e->ky, sV * total, "y"}, {&e->kz, sV * total, "z"}, {&e->kb, sV * total, "b"},
        {(void**)&e->partials, sizeof(double) * kMaxRed * e->nTiles, "partials"},
        {(void**)&e->counters, sizeof(unsigned) * members, "counters"},
        {(void**)&e->st, sizeof(BiState) * members, "state"},
        {(void**)&e->stSave, sizeof(BiState) * members, "saved state"},
        {(void**)&e->mask, sizeof(int) * members, "mask"},
        {(void**)&e->errmax, sizeof(unsigned long long) * members, "errmax"},
        {(void**)&e->flags, sizeof(int) * members, "flags"},
        {(void**)&e->flagsF, sizeof(int) * members, "factor flags"},
        {(void**)&e->flagsU, sizeof(int) * members, "update flags"},
        {(void**)&e->dtArr, sizeof(double) * members, "dt"},
    };
    for (const A& a : allocs) {
        if ((c = cudaMalloc(a.p, a.bytes)) != cudaSuccess) return failc(a.what);
        if ((c = cudaMemsetAsync(*a.p, 0, a.bytes, e->stream)) != cudaSuccess) return failc(a.what);
    }
    for (ewg_ensemble::TileList* tl : {&e->tlA, &e->tlB}) {
        if ((c = cudaMalloc(&tl->d, sizeof(int2) * e->nTiles)) != cudaSuccess) return failc("tile list");
        if ((c = cudaMalloc(&tl->dn, sizeof(int))) != cudaSuccess) return failc("tile list");
        if ((c = cudaMemsetAsync(tl->dn, 0, sizeof(int), e->stream)) != cudaSuccess) return failc("tile list");
        if ((c = cudaMallocHost(&tl->h, sizeof(int2) * e->nTiles)) != cudaSuccess) return failc("pinned tile list");
        if ((c = cudaMallocHost(&tl->hn, sizeof(int))) != cudaSuccess) return failc("pinned tile list");
        if ((c = cudaEventCreate(&tl->ev)) != cudaSuccess) return failc("event");
    }
    if ((c = cudaMallocHost(&e->hSt, sizeof(BiState) * members)) != cudaSuccess) return failc("pinned state");
    if ((c = cudaMallocHost(&e->hMask, sizeof(int) * members)) != cudaSuccess) return failc("pinned mask");
    if ((c = cudaMallocHost(&e->hErr, sizeof(unsigned long long) * members)) != cudaSuccess) return failc("pinned errmax");
    if ((c = cudaMallocHost(&e->hFlags, sizeof(int) * members)) != cudaSuccess) return failc("pinned flags");
    if ((c = cudaMallocHost(&e->hFlagsF, sizeof(int) * members)) != cudaSuccess) return failc("pinned flags");
    if ((c = cudaMallocHost(&e->hFlagsU, sizeof(int) * members)) != cudaSuccess) return failc("pinned flags");
    if ((c = cudaMallocHost(&e->hDt, sizeof(double) * members)) != cudaSuccess) return failc("pinned dt");
    if ((c = cudaMemcpyAsync(e->dm, e->hm.data(), sizeof(EnsMember) * members, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return failc("upload members");
    if ((c = cudaMemcpyAsync(e->geo, geoAll.data(), sizeof(FaceGeo) * geoAll.size(), cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
        return failc("upload geometry");
    for (int m = 0; m < members; ++m) {
        const EnsMember& em = e->hm[m];
        double* stage = reinterpret_cast<double*>(e->stage);
        if ((c = cudaMemcpyAsync(stage, perms[m], sizeof(double) * em.P.N, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess)
            return failc("upload perm");
        if ((c = layout_scalar_to_split(em.P, e->stream, stage, e->perm + em.off)) != cudaSuccess) return failc("perm layout");
        if ((c = layout_lens_flags(em.P, e->stream, e->lens + em.off)) != cudaSuccess) return failc("lens flags");
        // the host permeability is borrowed only for this call
        if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return failc("sync perm");
    }
    if (mixed) default_grids<float>(e);
    else default_grids<double>(e);
    if ((c = cudaStreamSynchronize(e->stream)) != cudaSuccess) return failc("sync create");
    *out = e;
    return EWG_OK;
}

int32_t ewg_ensemble_num_members(const ewg_ensemble* e) { return e ? e->M : 0; }

int64_t ewg_ensemble_num_cells(const ewg_ensemble* e, int32_t member) {
    if (!e) return 0;
    if (member < 0) return e->total;
    if (member >= e->M) return 0;
    return e->hm[member].P.N;
}

void* ewg_ensemble_get_stream(ewg_ensemble* e) { return e ? (void*)e->stream : nullptr; }

ewg_status ewg_ensemble_apply_initial_solution(ewg_ensemble* e) {
    if (check_ens(e)) return EWG_ERR_INVALID;
    std::vector<int> all(e->M);
    for (int m = 0; m < e->M; ++m) all[m] = m;
    ewg_status s = levels(e, all, 0);
    if (s) return s;
    return ens_fail(e, cudaStreamSynchronize(e->stream), "sync initial");
}

ewg_status ewg_ensemble_set_solution(ewg_ensemble* e, int32_t member, int32_t t, const double* x) {
    if (check_ens(e) || member < 0 || member >= e->M || (t != 0 && t != 1) || !x) return EWG_ERR_INVALID;
    const EnsMember& em = e->hm[member];
    cudaError_t c = cudaMemcpyAsync(e->stage, x, sizeof(double2) * em.P.N, cudaMemcpyHostToDevice, e->stream);
    if (c == cudaSuccess) c = layout_natural_to_split(em.P, e->stream, e->stage, (t == 0 ? e->x0 : e->x1) + em.off);
    if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
    if (c != cudaSuccess) return ens_fail(e, c, "set solution");
    if (t == 1) {
        // the old-time storage term follows solution(1)
        std::vector<int> one(1, member);
        ewg_status s = levels(e, one, 3);
        if (s) return s;
        return ens_fail(e, cudaStreamSynchronize(e->stream), "sync set solution");
    }
    return EWG_OK;
}

ewg_status ewg_ensemble_get_solution(ewg_ensemble* e, int32_t member, int32_t t, double* x) {
    if (check_ens(e) || member < 0 || member >= e->M || (t != 0 && t != 1) || !x) return EWG_ERR_INVALID;
    const EnsMember& em = e->hm[member];
    cudaError_t c = layout_split_to_natural(em.P, e->stream, (t == 0 ? e->x0 : e->x1) + em.off, e->stage);
    if (c == cudaSuccess) c = cudaMemcpyAsync(x, e->stage, sizeof(double2) * em.P.N, cudaMemcpyDeviceToHost, e->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
    return ens_fail(e, c, "get solution");
}

ewg_status ewg_ensemble_linearize(ewg_ensemble* e, const double* dt, double* max_norms) {
    if (check_ens(e) || !dt) return EWG_ERR_INVALID;
    std::vector<int> all(e->M);
    for (int m = 0; m < e->M; ++m) {
        if (!(dt[m] > 0)) { e->err = "dt must be positive"; return EWG_ERR_INVALID; }
        all[m] = m;
        e->hDt[m] = dt[m];
    }
    ewg_status s = e->precision == EWG_PRECISION_MIXED ? linearize_set<float>(e, all, true) : linearize_set<double>(e, all, true);
    if (s) return s;
    bool bad = false;
    for (int m = 0; m < e->M; ++m) {
        if (max_norms) max_norms[m] = (e->hFlags[m] & 1) ? INFINITY : err_of(e, m);
        bad = bad || (e->hFlags[m] & 1);
    }
    if (bad) { e->err = "non-finite residual"; return EWG_ERR_NONFINITE; }
    return EWG_OK;
}

ewg_status ewg_ensemble_get_residual(ewg_ensemble* e, int32_t member, double* r) {
    if (check_ens(e) || member < 0 || member >= e->M || !r) return EWG_ERR_INVALID;
    const EnsMember& em = e->hm[member];
    cudaError_t c = layout_split_to_natural(em.P, e->stream, e->r + em.off, e->stage);
    if (c == cudaSuccess) c = cudaMemcpyAsync(r, e->stage, sizeof(double2) * em.P.N, cudaMemcpyDeviceToHost, e->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(e->stream);
    return ens_fail(e, c, "get residual");
}

ewg_status ewg_ensemble_autotune(ewg_ensemble* e, const double* dt, const ewg_solve_opts* so) {
    if (check_ens(e) || !dt || !so) return EWG_ERR_INVALID;
    for (int m = 0; m < e->M; ++m)
        if (!(dt[m] > 0)) { e->err = "dt must be positive"; return EWG_ERR_INVALID; }
    return e->precision == EWG_PRECISION_MIXED ? autotune<float>(e, dt, so) : autotune<double>(e, dt, so);
}

ewg_status ewg_ensemble_get_launch_shapes(const ewg_ensemble* e, int32_t* grids, int32_t count, int32_t* assemble_variant) {
    if (!e || !grids || count < EC_NUM) return EWG_ERR_INVALID;
    for (int c = 0; c < EC_NUM; ++c) grids[c] = e->grid[c];
    if (assemble_variant) *assemble_variant = e->asmVariant;
    return EWG_OK;
}

ewg_status ewg_ensemble_advance(ewg_ensemble* e, int32_t steps, const double* dt, const ewg_newton_opts* no,
                                const ewg_solve_opts* so, ewg_ensemble_report* reports, ewg_ensemble_stats* stats) {
    if (check_ens(e) || !dt || !no || !so || steps < 1) return EWG_ERR_INVALID;
    if (so->precond != EWG_PRECOND_ILU0) { e->err = "ensembles use the block ILU(0) preconditioner"; return EWG_ERR_INVALID; }
    return e->precision == EWG_PRECISION_MIXED ? ensemble_advance<float>(e, steps, dt, no, so, reports, stats)
                                               : ensemble_advance<double>(e, steps, dt, no, so, reports, stats);
}

ewg_status ewg_ensemble_advance_device(ewg_ensemble* e, int32_t steps, const double* dt, const ewg_newton_opts* no,
                                       const ewg_solve_opts* so, ewg_ensemble_report* reports,
                                       ewg_ensemble_stats* stats) {
    if (check_ens(e) || !dt || !no || !so || steps < 1) return EWG_ERR_INVALID;
    if (so->precond != EWG_PRECOND_ILU0) { e->err = "ensembles use the block ILU(0) preconditioner"; return EWG_ERR_INVALID; }
    return e->precision == EWG_PRECISION_MIXED ? ensemble_advance_device<float>(e, steps, dt, no, so, reports, stats)
                                               : ensemble_advance_device<double>(e, steps, dt, no, so, reports, stats);
}

ewg_status ewg_ensemble_step(ewg_ensemble* e, const double* dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                             ewg_ensemble_report* reports, ewg_ensemble_stats* stats) {
    return ewg_ensemble_advance(e, 1, dt, no, so, reports, stats);
}

}  // extern "C"
