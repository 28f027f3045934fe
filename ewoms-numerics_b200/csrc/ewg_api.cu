// C ABI of libewg.so (include/ewg.h): context lifecycle, host <-> device layout conversion, the
// BCRS view of the band Jacobian, and the Newton driver that replays NewtonMethod::apply
// (nonlinear/newtonmethod.hh:308-517) on device-resident data.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

#include "ewg_internal.cuh"

namespace {
thread_local std::string g_createError;
}

namespace ewg {

constexpr int kApiBlock = 256;

ewg_status cuda_fail(ewg_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EWG_OK;
    ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
    return EWG_ERR_CUDA;
}

const char* const kKernelNames[K_NUM_KERNELS] = {
    "intensive", "assemble", "storage", "initial", "layout",
    "diag_inverse", "ilu_black_factor", "ilu_black_apply", "ilu_red_apply", "jacobi_apply",
    "spmv", "bicg_init", "bicg_p", "bicg_spmv_alpha", "bicg_hs", "bicg_spmv_omega", "bicg_xr",
    "to_float", "defect_accumulate", "defect_residual", "newton_update", "bcrs",
    "bicg_true_residual", "b8_layout", "b8_factor", "b8_forward", "b8_backward"};

void prof_flush(ewg_ctx* ctx) {
    Profiler& pr = ctx->prof;
    for (int q = 0; q < pr.npend; ++q) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pr.ev[2 * q], pr.ev[2 * q + 1]) == cudaSuccess) pr.ms[pr.pendId[q]] += ms;
    }
    pr.npend = 0;
}

void prof_begin(ewg_ctx* ctx, int id) {
    Profiler& pr = ctx->prof;
    pr.pendingTimed = pr.on && (pr.launches[id] % pr.period) == 0;
    if (!pr.pendingTimed) return;
    if (pr.npend == Profiler::kPool) {
        cudaStreamSynchronize(ctx->stream);
        prof_flush(ctx);
    }
    cudaEventRecord(pr.ev[2 * pr.npend], ctx->stream);
    pr.pendId[pr.npend] = id;
}

void prof_end(ewg_ctx* ctx, int id) {
    Profiler& pr = ctx->prof;
    pr.launches[id] += 1;
    if (!pr.pendingTimed) return;
    pr.pendingTimed = false;
    pr.sampled[id] += 1;
    cudaEventRecord(pr.ev[2 * pr.npend + 1], ctx->stream);
    pr.npend += 1;
}

int grid_size_for(ewg_ctx* ctx, const void* kernel, int block, size_t smem) {
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, block, smem) != cudaSuccess || perSM < 1)
        perSM = 1;
    int64_t need = (ctx->P.N + block - 1) / block;
    int64_t full = (int64_t)ctx->numSMs * perSM;
    return (int)(need < full ? (need > 0 ? need : 1) : full);
}

// ---- material-law constants (RegularizedVanGenuchtenParams / RegularizedBrooksCoreyParams) ----

static double vgPcnwHost(const LawDev& L, double Se) {
    return std::pow(std::pow(Se, L.negInvM) - 1.0, L.invN) / L.alpha;
}
// central finite difference with eps 1e-7 (RegularizedVanGenuchtenParams::dPcnw_dSw_)
static double vgDPcFdHost(const LawDev& L, double Sw) {
    const double eps = 1e-7;
    double delta = 0.0, pc1, pc2;
    if (Sw + eps < 1.0) { pc2 = vgPcnwHost(L, Sw + eps); delta += eps; } else pc2 = vgPcnwHost(L, Sw);
    if (Sw - eps > 0.0) { pc1 = vgPcnwHost(L, Sw - eps); delta += eps; } else pc1 = vgPcnwHost(L, Sw);
    return (pc2 - pc1) / delta;
}
static double bcDPcHost(const LawDev& L, double pe, double lambda, double Sw) {
    (void)L;
    return -pe / lambda * std::pow(Sw, -1.0 / lambda - 1.0);
}

static LawDev make_law(const ewg_material& m) {
    LawDev L;
    memset(&L, 0, sizeof(L));
    L.kind = m.law;
    L.swr = m.swr;
    L.snr = m.snr;
    L.den = 1.0 - (m.swr + m.snr);
    if (m.law == EWG_LAW_VAN_GENUCHTEN) {
        L.alpha = m.vg_alpha;
        L.n = m.vg_n;
        L.m = 1.0 - 1.0 / m.vg_n;
        L.negInvM = -1.0 / L.m;
        L.invN = 1.0 / L.n;
        L.invM = 1.0 / L.m;
        L.twoM = 2 * L.m;
        L.pcLowSw = 0.01;
        L.pcHighSw = 0.99;
        L.pcLow = vgPcnwHost(L, L.pcLowSw);
        L.pcSlopeLow = vgDPcFdHost(L, L.pcLowSw);
        const double pcHigh = vgPcnwHost(L, L.pcHighSw);
        L.m1High = (0.0 - pcHigh) / (1.0 - L.pcHighSw) * 2;
        const double slopeHigh = 2 * (0.0 - pcHigh) / (1.0 - L.pcHighSw);
        const double mTh = vgDPcFdHost(L, L.pcHighSw);
        L.spX0 = L.pcHighSw;
        L.spH = 1.0 - L.pcHighSw;
        L.spY0 = pcHigh;
        L.spY1 = 0.0;
        L.spHM0 = L.spH * mTh;
        L.spHM1 = L.spH * slopeHigh;
    } else {
        const double pe = m.bc_entry_pressure, lam = m.bc_lambda;
        L.pe = pe;
        L.negInvLambda = -1.0 / lam;
        L.krwExp = 2.0 / lam + 3;
        L.krnExp = 2.0 / lam + 1;
        L.bcLowSw = 0.01;
        L.bcPcLow = pe * std::pow(0.01, -1.0 / lam);
        L.bcSlopeLow = bcDPcHost(L, pe, lam, 0.01);
        L.bcSlopeOne = bcDPcHost(L, pe, lam, 1.0);
    }
    return L;
}

void build_phys(Phys& P, const ewg_grid* g, const ewg_problem* p) {
    memset(&P, 0, sizeof(P));
    P.dim = g->dim;
    P.nx = g->nx;
    P.ny = g->ny;
    P.nz = g->dim == 3 ? g->nz : 1;
    set_index_constants(P);
    P.L[0] = g->lx;
    P.L[1] = g->ly;
    P.L[2] = g->dim == 3 ? g->lz : 1.0;
    P.kOrigin = g->dim == 3 ? g->k_origin : 0;
    const int n[3] = {P.nx, P.ny, P.nz};
    for (int a = 0; a < 3; ++a) P.h[a] = P.L[a] / n[a];
    if (P.dim == 2) {
        P.vol = P.h[0] * P.h[1];
        P.area[0] = P.h[1];
        P.area[1] = P.h[0];
        P.area[2] = 0.0;
    } else {
        P.vol = P.h[0] * P.h[1] * P.h[2];
        P.area[0] = P.h[1] * P.h[2];
        P.area[1] = P.h[0] * P.h[2];
        P.area[2] = P.h[0] * P.h[1];
    }
    P.porosity = p->porosity;
    P.rho[0] = p->rho_w;
    P.rho[1] = p->rho_n;
    P.mu[0] = p->mu_w;
    P.mu[1] = p->mu_n;
    P.g = p->gravity;
    P.pRef = p->p_ref;
    P.leftScale = p->left_pressure_scale;
    P.inletXlo = p->inlet_x_lo;
    P.inletXhi = p->inlet_x_hi;
    P.inletZlo = p->inlet_z_lo;
    P.inletZhi = p->inlet_z_hi;
    P.inletRate = p->inlet_rate;
    for (int a = 0; a < 3; ++a) {
        P.lensLo[a] = p->lens_lo[a];
        P.lensHi[a] = p->lens_hi[a];
    }
    P.eps = p->eps;
    for (int a = 0; a < 3; ++a)
        for (int ph = 0; ph < 2; ++ph) P.rhoArea[a][ph] = P.rho[ph] * P.area[a];
    P.invVol = 1.0 / P.vol;
    P.law[0] = make_law(p->outer);
    P.law[1] = make_law(p->lens);
}

// ---- layout kernels -------------------------------------------------------------------------

__global__ void k_natural_to_split(const __grid_constant__ Phys P, const double2* __restrict__ nat, double2* __restrict__ spl) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x)
        spl[split_of(P, c)] = nat[c];
}
__global__ void k_split_to_natural(const __grid_constant__ Phys P, const double2* __restrict__ spl, double2* __restrict__ nat) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x)
        nat[c] = spl[split_of(P, c)];
}
__global__ void k_scalar_to_split(const __grid_constant__ Phys P, const double* __restrict__ nat, double* __restrict__ spl) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x)
        spl[split_of(P, c)] = nat[c];
}
__global__ void k_lens_flags(const __grid_constant__ Phys P, uint8_t* __restrict__ lens) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        const int col = s >= P.Nh ? 1 : 0;
        const CellIdx ci = cell_of(P, col, s - col * P.Nh);
        const int idx[3] = {ci.i, ci.j, ci.k};
        bool in = true;
        for (int a = 0; a < P.dim; ++a) {
            double x = (idx[a] + (a == 2 ? P.kOrigin : 0) + 0.5) * P.h[a];
            if (x < P.lensLo[a] - P.eps || x > P.lensHi[a] + P.eps) in = false;
        }
        lens[s] = in ? 1 : 0;
    }
}

// launchers of the layout kernels for a problem that has no context (ensemble members)
static int layout_grid(const Phys& P) {
    int64_t g = (P.N + kApiBlock - 1) / kApiBlock;
    return (int)(g < 4096 ? (g > 0 ? g : 1) : 4096);
}
cudaError_t layout_natural_to_split(const Phys& P, cudaStream_t st, const double2* nat, double2* spl) {
    k_natural_to_split<<<layout_grid(P), kApiBlock, 0, st>>>(P, nat, spl);
    return cudaGetLastError();
}
cudaError_t layout_split_to_natural(const Phys& P, cudaStream_t st, const double2* spl, double2* nat) {
    k_split_to_natural<<<layout_grid(P), kApiBlock, 0, st>>>(P, spl, nat);
    return cudaGetLastError();
}
cudaError_t layout_scalar_to_split(const Phys& P, cudaStream_t st, const double* nat, double* spl) {
    k_scalar_to_split<<<layout_grid(P), kApiBlock, 0, st>>>(P, nat, spl);
    return cudaGetLastError();
}
cudaError_t layout_lens_flags(const Phys& P, cudaStream_t st, uint8_t* lens) {
    k_lens_flags<<<layout_grid(P), kApiBlock, 0, st>>>(P, lens);
    return cudaGetLastError();
}

// p_c, lambda_w, lambda_n of every cell (split-order cache planes 0, 2, 4) in natural order
__global__ void k_iq_natural(const __grid_constant__ Phys P, const double* __restrict__ iq, double* __restrict__ out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = split_of(P, c);
        out[3 * c] = iq[s];
        out[3 * c + 1] = iq[2 * P.N + s];
        out[3 * c + 2] = iq[4 * P.N + s];
    }
}

// natural row c of the reference BCRS, columns ascending: the band of each entry
__device__ __forceinline__ int band_for_column(const Phys& P, int64_t c, int64_t col) {
    if (col < 0 || col >= P.N) return -1;
    const int64_t pl = (int64_t)P.nx * P.ny;
    const int ci = (int)(c % P.nx), cj = (int)((c / P.nx) % P.ny), ck = (int)(c / pl);
    const int qi = (int)(col % P.nx), qj = (int)((col / P.nx) % P.ny), qk = (int)(col / pl);
    const int di = qi - ci, dj = qj - cj, dk = qk - ck;
    const int nz = (di != 0) + (dj != 0) + (dk != 0);
    if (nz == 0) return 0;
    if (nz != 1) return -1;
    if (di == -1) return 1;
    if (di == 1) return 2;
    if (dj == -1) return 3;
    if (dj == 1) return 4;
    if (dk == -1 && P.dim == 3) return 5;
    if (dk == 1 && P.dim == 3) return 6;
    return -1;
}

template <bool EXPORT>
__global__ void k_bcrs_blocks(const __grid_constant__ Phys P, const int32_t* __restrict__ rowPtr,
                              const int32_t* __restrict__ colIdx, double* __restrict__ J, double* __restrict__ blocks,
                              int* bad) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = split_of(P, c);
        for (int32_t q = rowPtr[c]; q < rowPtr[c + 1]; ++q) {
            const int band = band_for_column(P, c, colIdx[q]);
            if (band < 0) { atomicOr(bad, 1); continue; }
            double* base = J + (int64_t)band * 4 * P.N + s;
            for (int t = 0; t < 4; ++t) {
                if (EXPORT) blocks[4 * (int64_t)q + t] = base[t * P.N];
                else base[t * P.N] = blocks[4 * (int64_t)q + t];
            }
        }
    }
}

static int lgrid(ewg_ctx* ctx, const void* k) { return grid_size_for(ctx, k, kApiBlock); }

ewg_status to_split(ewg_ctx* ctx, const double* host, double2* dev) {
    cudaError_t e;
    const size_t bytes = sizeof(double2) * ctx->P.N;
    if ((e = cudaMemcpyAsync(ctx->d_stage, host, bytes, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "H2D");
    ctx->h2dBytes += bytes;
    EWG_LAUNCH(ctx, K_LAYOUT, k_natural_to_split, lgrid(ctx, (const void*)k_natural_to_split), kApiBlock, ctx->P, ctx->d_stage, dev);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "natural_to_split");
    return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync H2D");
}

ewg_status from_split(ewg_ctx* ctx, const double2* dev, double* host) {
    cudaError_t e;
    const size_t bytes = sizeof(double2) * ctx->P.N;
    EWG_LAUNCH(ctx, K_LAYOUT, k_split_to_natural, lgrid(ctx, (const void*)k_split_to_natural), kApiBlock, ctx->P, dev, ctx->d_stage);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "split_to_natural");
    if ((e = cudaMemcpyAsync(host, ctx->d_stage, bytes, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "D2H");
    ctx->d2hBytes += bytes;
    return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync D2H");
}

// reference BCRS pattern of the structured grid (createMatrix_: {i} + face neighbours, sorted)
static void host_pattern(const Phys& P, std::vector<int32_t>& rp, std::vector<int32_t>& ci) {
    rp.assign(P.N + 1, 0);
    ci.clear();
    ci.reserve((size_t)P.N * P.nb);
    const int64_t pl = (int64_t)P.nx * P.ny;
    for (int64_t c = 0; c < P.N; ++c) {
        const int i = (int)(c % P.nx);
        const int j = (int)((c / P.nx) % P.ny);
        const int k = (int)(c / pl);
        if (P.dim == 3 && k > 0) ci.push_back((int32_t)(c - pl));
        if (j > 0) ci.push_back((int32_t)(c - P.nx));
        if (i > 0) ci.push_back((int32_t)(c - 1));
        ci.push_back((int32_t)c);
        if (i < P.nx - 1) ci.push_back((int32_t)(c + 1));
        if (j < P.ny - 1) ci.push_back((int32_t)(c + P.nx));
        if (P.dim == 3 && k < P.nz - 1) ci.push_back((int32_t)(c + pl));
        rp[c + 1] = (int32_t)ci.size();
    }
}

}  // namespace ewg

using namespace ewg;

static ewg_status check_ctx(ewg_ctx* ctx) { return ctx ? EWG_OK : EWG_ERR_INVALID; }

extern "C" {

int32_t ewg_abi_version(void) { return EWG_ABI_VERSION; }
const char* ewg_create_error(void) { return g_createError.c_str(); }
const char* ewg_last_error(const ewg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }
int64_t ewg_num_cells(const ewg_ctx* ctx) { return ctx ? ctx->P.N : 0; }
int64_t ewg_num_blocks(const ewg_ctx* ctx) { return ctx ? ctx->nnzb : 0; }

void ewg_default_solve_opts(ewg_solve_opts* o) {
    memset(o, 0, sizeof(*o));
    o->precond = EWG_PRECOND_ILU0;
    o->precision = EWG_PRECISION_FP64;
    o->linear_solver_tolerance = 1e-3;
    o->linear_solver_abs_tolerance = 1e-10;  // NewtonTolerance / 100
    o->linear_solver_max_error = 1e7;
    o->linear_solver_max_iterations = 1000;
    o->preconditioner_relaxation = 1.0;
    o->defect_tolerance = 0.0;
    o->inner_tolerance = 1e-4;
    o->max_defect_iterations = 50;
    o->check_interval = 0;
    o->restart_on_breakdown = 1;
    o->verify_true_residual = 1;
    o->ilu_ordering = EWG_ILU_ORDER_AUTO;
}

void* ewg_get_stream(ewg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
int32_t ewg_profile_num_kernels(void) { return K_NUM_KERNELS; }
const char* ewg_profile_kernel_name(int32_t id) { return id >= 0 && id < K_NUM_KERNELS ? kKernelNames[id] : ""; }

ewg_status ewg_profile_enable(ewg_ctx* ctx, int32_t on) {
    if (!ctx) return EWG_ERR_INVALID;
    Profiler& pr = ctx->prof;
    if (on && !pr.created) {
        for (int q = 0; q < 2 * Profiler::kPool; ++q) {
            cudaError_t e = cudaEventCreate(&pr.ev[q]);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "profiler events");
        }
        pr.created = true;
    }
    cudaStreamSynchronize(ctx->stream);
    prof_flush(ctx);
    pr.on = on != 0;
    pr.period = on > 1 ? on : 1;
    return EWG_OK;
}

ewg_status ewg_profile_reset(ewg_ctx* ctx) {
    if (!ctx) return EWG_ERR_INVALID;
    cudaStreamSynchronize(ctx->stream);
    prof_flush(ctx);
    for (int k = 0; k < K_NUM_KERNELS; ++k) {
        ctx->prof.ms[k] = 0.0;
        ctx->prof.launches[k] = 0;
        ctx->prof.sampled[k] = 0;
    }
    return EWG_OK;
}

ewg_status ewg_profile_get(ewg_ctx* ctx, int32_t id, double* msTotal, int64_t* launches) {
    if (!ctx || id < 0 || id >= K_NUM_KERNELS) return EWG_ERR_INVALID;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "profile sync");
    prof_flush(ctx);
    // with a sampling period the timed launches stand for all launches of the class
    const Profiler& pr = ctx->prof;
    if (msTotal) *msTotal = pr.sampled[id] ? pr.ms[id] * (double)pr.launches[id] / (double)pr.sampled[id] : 0.0;
    if (launches) *launches = ctx->prof.launches[id];
    return EWG_OK;
}

void ewg_default_newton_opts(ewg_newton_opts* o) {
    memset(o, 0, sizeof(*o));
    o->newton_tolerance = 1e-8;
    o->newton_max_error = 1e100;
    o->newton_max_iterations = 18;
    o->newton_target_iterations = 10;
    o->verbose = 0;
}

ewg_status ewg_create(const ewg_grid* grid, const ewg_problem* problem, const double* perm, ewg_ctx** out) {
    g_createError.clear();
    if (!grid || !problem || !perm || !out) { g_createError = "null argument"; return EWG_ERR_INVALID; }
    *out = nullptr;
    if (grid->dim != 2 && grid->dim != 3) { g_createError = "dim must be 2 or 3"; return EWG_ERR_INVALID; }
    const int nz = grid->dim == 3 ? grid->nz : 1;
    if (grid->nx < 2 || grid->ny < 1 || nz < 1 || (grid->nx & 1)) {
        g_createError = "nx must be even and >= 2 (red-black split storage), ny, nz >= 1";
        return EWG_ERR_INVALID;
    }
    if ((int64_t)grid->nx * grid->ny * nz >= (int64_t)1 << 31) { g_createError = "grid too large for int32 BCRS indices"; return EWG_ERR_INVALID; }
    if (grid->dim == 3 && grid->k_origin < 0) { g_createError = "k_origin must be >= 0"; return EWG_ERR_INVALID; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        g_createError = "no CUDA device";
        return EWG_ERR_NO_DEVICE;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10) {
        g_createError = "device is not sm_100 (B200)";
        return EWG_ERR_NO_DEVICE;
    }
    ewg_ctx* ctx = new ewg_ctx();
    ctx->device = dev;
    ctx->numSMs = prop.multiProcessorCount;
    build_phys(ctx->P, grid, problem);
    const Phys& P = ctx->P;
    cudaError_t e = cudaSuccess;
    auto fail = [&](const char* what) {
        g_createError = std::string(what) + ": " + cudaGetErrorString(e);
        ewg_destroy(ctx);
        return EWG_ERR_CUDA;
    };
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail("stream");
    if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess) return fail("event");
    if ((e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) return fail("event");
    const size_t nv = sizeof(double2) * P.N;
    if ((e = cudaMalloc(&ctx->x0, nv)) != cudaSuccess) return fail("alloc x0");
    if ((e = cudaMalloc(&ctx->x1, nv)) != cudaSuccess) return fail("alloc x1");
    if ((e = cudaMalloc(&ctx->sold, nv)) != cudaSuccess) return fail("alloc storage");
    if ((e = cudaMalloc(&ctx->r, nv)) != cudaSuccess) return fail("alloc r");
    if ((e = cudaMalloc(&ctx->dx, nv)) != cudaSuccess) return fail("alloc dx");
    if ((e = cudaMalloc(&ctx->d_stage, nv)) != cudaSuccess) return fail("alloc staging");
    if ((e = cudaMalloc(&ctx->perm, sizeof(double) * P.N)) != cudaSuccess) return fail("alloc perm");
    if ((e = cudaMalloc(&ctx->lens, P.N)) != cudaSuccess) return fail("alloc lens");
    if ((e = cudaMalloc(&ctx->iq, sizeof(double) * 6 * P.N)) != cudaSuccess) return fail("alloc iq");
    if ((e = cudaMalloc(&ctx->J, sizeof(double) * 4 * P.nb * P.N)) != cudaSuccess) return fail("alloc J");
    if ((e = cudaMemsetAsync(ctx->J, 0, sizeof(double) * 4 * P.nb * P.N, ctx->stream)) != cudaSuccess) return fail("zero J");
    if ((e = cudaMalloc(&ctx->d_errmax, sizeof(unsigned long long))) != cudaSuccess) return fail("alloc errmax");
    if ((e = cudaMalloc(&ctx->d_flags, sizeof(int) * 4)) != cudaSuccess) return fail("alloc flags");
    if ((e = cudaMemsetAsync(ctx->x0, 0, nv, ctx->stream)) != cudaSuccess) return fail("zero");
    if ((e = cudaMemsetAsync(ctx->x1, 0, nv, ctx->stream)) != cudaSuccess) return fail("zero");
    if ((e = cudaMemsetAsync(ctx->sold, 0, nv, ctx->stream)) != cudaSuccess) return fail("zero");
    if ((e = cudaMemsetAsync(ctx->r, 0, nv, ctx->stream)) != cudaSuccess) return fail("zero");
    if ((e = cudaMemsetAsync(ctx->dx, 0, nv, ctx->stream)) != cudaSuccess) return fail("zero");
    // permeability (natural -> split) and lens flags
    double* stage = nullptr;
    if ((e = cudaMalloc(&stage, sizeof(double) * P.N)) != cudaSuccess) return fail("alloc stage");
    e = cudaMemcpyAsync(stage, perm, sizeof(double) * P.N, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        EWG_LAUNCH(ctx, K_LAYOUT, k_scalar_to_split, lgrid(ctx, (const void*)k_scalar_to_split), kApiBlock, P, stage, ctx->perm);
        EWG_LAUNCH(ctx, K_LAYOUT, k_lens_flags, lgrid(ctx, (const void*)k_lens_flags), kApiBlock, P, ctx->lens);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    cudaFree(stage);
    if (e != cudaSuccess) return fail("upload permeability");
    {
        ewg_status bst = compute_boundary_constants(ctx);
        if (bst == EWG_OK) bst = build_interior_tables(ctx);
        if (bst != EWG_OK) { g_createError = ctx->err; ewg_destroy(ctx); return bst; }
    }
    // reference BCRS pattern
    std::vector<int32_t> rp, ci;
    host_pattern(P, rp, ci);
    ctx->nnzb = (int64_t)ci.size();
    if ((e = cudaMalloc(&ctx->d_rowPtr, sizeof(int32_t) * rp.size())) != cudaSuccess) return fail("alloc rowptr");
    if ((e = cudaMalloc(&ctx->d_colIdx, sizeof(int32_t) * ci.size())) != cudaSuccess) return fail("alloc colidx");
    if ((e = cudaMemcpyAsync(ctx->d_rowPtr, rp.data(), sizeof(int32_t) * rp.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail("upload rowptr");
    if ((e = cudaMemcpyAsync(ctx->d_colIdx, ci.data(), sizeof(int32_t) * ci.size(), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return fail("upload colidx");
    // everything above is ordered on the context stream; finish it before returning
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return fail("sync create");
    *out = ctx;
    return EWG_OK;
}

void ewg_destroy(ewg_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    solver_free(ctx);
    void* ps[] = {ctx->x0, ctx->x1, ctx->sold, ctx->r, ctx->dx, ctx->d_stage, ctx->perm, ctx->lens, ctx->iq, ctx->J, ctx->J32, ctx->geo,
                  ctx->d_errmax, ctx->d_flags, ctx->d_rowPtr, ctx->d_colIdx};
    for (void* p : ps) if (p) cudaFree(p);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->prof.created)
        for (int q = 0; q < 2 * Profiler::kPool; ++q) cudaEventDestroy(ctx->prof.ev[q]);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

ewg_status ewg_set_solution(ewg_ctx* ctx, int32_t t, const double* x) {
    if (check_ctx(ctx) || !x || (t != 0 && t != 1)) return EWG_ERR_INVALID;
    ewg_status st = to_split(ctx, x, t == 0 ? ctx->x0 : ctx->x1);
    if (st) return st;
    if (t == 1) {
        if ((st = launch_storage(ctx, ctx->x1, ctx->sold))) return st;
        return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync storage");
    }
    return EWG_OK;
}

ewg_status ewg_get_solution(ewg_ctx* ctx, int32_t t, double* x) {
    if (check_ctx(ctx) || !x || (t != 0 && t != 1)) return EWG_ERR_INVALID;
    return from_split(ctx, t == 0 ? ctx->x0 : ctx->x1, x);
}

ewg_status ewg_apply_initial_solution(ewg_ctx* ctx) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    ewg_status st = launch_initial_solution(ctx, ctx->x0);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(ctx->x1, ctx->x0, sizeof(double2) * ctx->P.N, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy x1");
    if ((st = launch_storage(ctx, ctx->x1, ctx->sold))) return st;
    return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync initial");
}

ewg_status ewg_advance_time_level(ewg_ctx* ctx) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(ctx->x1, ctx->x0, sizeof(double2) * ctx->P.N, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "advance");
    ewg_status st = launch_storage(ctx, ctx->x1, ctx->sold);
    if (st) return st;
    return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync advance");
}

ewg_status ewg_restore_time_level(ewg_ctx* ctx) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(ctx->x0, ctx->x1, sizeof(double2) * ctx->P.N, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "restore");
    return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync restore");
}

static ewg_status ensure_j32(ewg_ctx* ctx) {
    if (ctx->J32) return EWG_OK;
    const size_t bytes = sizeof(float) * 4 * ctx->P.nb * ctx->P.N;
    cudaError_t e = cudaMalloc(&ctx->J32, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "alloc J32");
    e = cudaMemsetAsync(ctx->J32, 0, bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return cuda_fail(ctx, e, "zero J32");
}

// ImmiscibleModel::updateBegin (immisciblemodel.hh:278-293): p_w of the first DOF of solution(0)
// (natural cell 0 is split position 0). Only the finite-difference linearizer uses it.
static ewg_status update_reference_pressure(ewg_ctx* ctx, bool force) {
    if (!force && (ctx->localLinearizer != EWG_LOCAL_LINEARIZER_FD || ctx->refPressure > 0)) return EWG_OK;
    double p = 0.0;
    cudaError_t e = cudaMemcpyAsync(&p, &ctx->x0[0].x, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "read reference pressure");
    if (!(p > 0) || !std::isfinite(p)) {
        ctx->err = "finite-difference linearizer: the reference pressure (p_w of cell 0) must be positive";
        return EWG_ERR_NONFINITE;
    }
    ctx->refPressure = p;
    return EWG_OK;
}

static ewg_status linearize_impl(ewg_ctx* ctx, double dt, ewg_lin_report* rep) {
    if (!(dt > 0)) { ctx->err = "dt must be positive"; return EWG_ERR_INVALID; }
    if (ctx->jacPrecision == EWG_PRECISION_MIXED) {
        ewg_status st = ensure_j32(ctx);
        if (st) return st;
    }
    cudaEventRecord(ctx->ev0, ctx->stream);
    double err = 0;
    int bad = 0;
    ewg_status st = launch_linearize(ctx, dt, true, ctx->x0, ctx->r, &err, &bad);
    if (st) return st;
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaEventSynchronize(ctx->ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->jacFromLinearizer = true;
    ctx->iluValid = false;
    if (rep) {
        rep->error = bad ? INFINITY : err;
        rep->nonfinite = bad;
        rep->seconds = ms * 1e-3;
    }
    if (bad) { ctx->err = "non-finite residual"; return EWG_ERR_NONFINITE; }
    return EWG_OK;
}

ewg_status ewg_linearize(ewg_ctx* ctx, double dt, ewg_lin_report* rep) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    // a context that never ran updateBegin takes the reference pressure of the current iterate
    ewg_status st = update_reference_pressure(ctx, false);
    if (st) return st;
    return linearize_impl(ctx, dt, rep);
}

ewg_status ewg_update_begin(ewg_ctx* ctx) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    return update_reference_pressure(ctx, true);
}

ewg_status ewg_set_reference_pressure(ewg_ctx* ctx, double p_ref) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    if (!(p_ref > 0) || !std::isfinite(p_ref)) {
        ctx->err = "set_reference_pressure: p_ref must be positive and finite";
        return EWG_ERR_INVALID;
    }
    ctx->refPressure = p_ref;
    return EWG_OK;
}

ewg_status ewg_get_intensive_quantities(ewg_ctx* ctx, double* out) {
    if (check_ctx(ctx) || !out) return EWG_ERR_INVALID;
    ewg_status st = launch_intensive(ctx, ctx->x0);
    if (st) return st;
    double* d = nullptr;
    const size_t bytes = sizeof(double) * 3 * ctx->P.N;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "alloc intensive output");
    k_iq_natural<<<lgrid(ctx, (const void*)k_iq_natural), kApiBlock, 0, ctx->stream>>>(ctx->P, ctx->iq, d);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) ctx->d2hBytes += bytes;
    cudaFree(d);
    return cuda_fail(ctx, e, "intensive quantities");
}

ewg_status ewg_set_local_linearizer(ewg_ctx* ctx, int32_t kind, int32_t method) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    if (kind != EWG_LOCAL_LINEARIZER_AD && kind != EWG_LOCAL_LINEARIZER_FD) {
        ctx->err = "unknown local linearizer";
        return EWG_ERR_INVALID;
    }
    if (method < -1 || method > 1) {
        ctx->err = "NumericDifferenceMethod must be -1, 0 or +1";
        return EWG_ERR_INVALID;
    }
    ctx->localLinearizer = kind;
    ctx->fdMethod = method;
    ctx->jacFromLinearizer = false;
    ctx->iluValid = false;
    return EWG_OK;
}

ewg_status ewg_get_residual(ewg_ctx* ctx, double* r) {
    if (check_ctx(ctx) || !r) return EWG_ERR_INVALID;
    return from_split(ctx, ctx->r, r);
}

ewg_status ewg_get_jacobian_bcrs(ewg_ctx* ctx, int32_t* rowPtr, int32_t* colIdx, double* blocks) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    cudaError_t e;
    const Phys& P = ctx->P;
    if (rowPtr && (e = cudaMemcpyAsync(rowPtr, ctx->d_rowPtr, sizeof(int32_t) * (P.N + 1), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "rowptr");
    if (rowPtr) ctx->d2hBytes += sizeof(int32_t) * (P.N + 1);
    if (colIdx && (e = cudaMemcpyAsync(colIdx, ctx->d_colIdx, sizeof(int32_t) * ctx->nnzb, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
        return cuda_fail(ctx, e, "colidx");
    if (colIdx) ctx->d2hBytes += sizeof(int32_t) * ctx->nnzb;
    if (!blocks) return cuda_fail(ctx, cudaStreamSynchronize(ctx->stream), "sync pattern");
    if (ctx->jacPrecision != EWG_PRECISION_FP64) { ctx->err = "BCRS export needs the FP64 Jacobian"; return EWG_ERR_INVALID; }
    double* tmp = nullptr;
    if ((e = cudaMalloc(&tmp, sizeof(double) * 4 * ctx->nnzb)) != cudaSuccess) return cuda_fail(ctx, e, "alloc export");
    cudaMemsetAsync(ctx->d_flags, 0, sizeof(int), ctx->stream);
    EWG_LAUNCH(ctx, K_BCRS, k_bcrs_blocks<true>, lgrid(ctx, (const void*)k_bcrs_blocks<true>), kApiBlock, P, ctx->d_rowPtr, ctx->d_colIdx, ctx->J, tmp, ctx->d_flags);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(blocks, tmp, sizeof(double) * 4 * ctx->nnzb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) ctx->d2hBytes += sizeof(double) * 4 * ctx->nnzb;
    cudaFree(tmp);
    return cuda_fail(ctx, e, "export blocks");
}

ewg_status ewg_set_matrix_bcrs(ewg_ctx* ctx, const int32_t* rowPtr, const int32_t* colIdx, const double* blocks) {
    if (check_ctx(ctx) || !rowPtr || !colIdx || !blocks) return EWG_ERR_INVALID;
    const Phys& P = ctx->P;
    std::vector<int32_t> rp, ci;
    host_pattern(P, rp, ci);
    if (memcmp(rp.data(), rowPtr, sizeof(int32_t) * rp.size()) != 0 ||
        memcmp(ci.data(), colIdx, sizeof(int32_t) * ci.size()) != 0) {
        ctx->err = "matrix pattern differs from the structured-grid pattern";
        return EWG_ERR_INVALID;
    }
    cudaError_t e;
    double* tmp = nullptr;
    if ((e = cudaMalloc(&tmp, sizeof(double) * 4 * ctx->nnzb)) != cudaSuccess) return cuda_fail(ctx, e, "alloc import");
    // stream-ordered: a plain cudaMemcpy from pageable memory may return before its DMA lands,
    // and the legacy stream does not order the non-blocking context stream
    e = cudaMemcpyAsync(tmp, blocks, sizeof(double) * 4 * ctx->nnzb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        ctx->h2dBytes += sizeof(double) * 4 * ctx->nnzb;
        EWG_LAUNCH(ctx, K_BCRS, k_bcrs_blocks<false>, lgrid(ctx, (const void*)k_bcrs_blocks<false>), kApiBlock, P, ctx->d_rowPtr, ctx->d_colIdx, ctx->J, tmp, ctx->d_flags);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    cudaFree(tmp);
    ctx->jacPrecision = EWG_PRECISION_FP64;
    ctx->iluValid = false;
    return cuda_fail(ctx, e, "import blocks");
}

ewg_status ewg_set_residual(ewg_ctx* ctx, const double* b) {
    if (check_ctx(ctx) || !b) return EWG_ERR_INVALID;
    return to_split(ctx, b, ctx->r);
}

ewg_status ewg_transfer_counters(ewg_ctx* ctx, int32_t reset, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    if (h2d_bytes) *h2d_bytes = ctx->h2dBytes;
    if (d2h_bytes) *d2h_bytes = ctx->d2hBytes;
    if (reset) ctx->h2dBytes = ctx->d2hBytes = 0;
    return EWG_OK;
}

ewg_status ewg_residual_norm(ewg_ctx* ctx, const double* x, double dt, double* maxNorm) {
    if (check_ctx(ctx) || !x || !maxNorm) return EWG_ERR_INVALID;
    cudaError_t e;
    double2* xs = nullptr;
    double2* rs = nullptr;
    if ((e = cudaMalloc(&xs, sizeof(double2) * ctx->P.N)) != cudaSuccess) return cuda_fail(ctx, e, "alloc");
    if ((e = cudaMalloc(&rs, sizeof(double2) * ctx->P.N)) != cudaSuccess) { cudaFree(xs); return cuda_fail(ctx, e, "alloc"); }
    ewg_status st = to_split(ctx, x, xs);
    int bad = 0;
    double v = 0;
    if (!st) st = launch_linearize(ctx, dt, false, xs, rs, &v, &bad);
    cudaFree(xs);
    cudaFree(rs);
    if (st) return st;
    *maxNorm = bad ? INFINITY : v;
    return EWG_OK;
}

ewg_status ewg_solve(ewg_ctx* ctx, const ewg_solve_opts* o, ewg_solve_report* rep) {
    if (check_ctx(ctx) || !o || !rep) return EWG_ERR_INVALID;
    return solver_solve(ctx, o, rep);
}

ewg_status ewg_get_update(ewg_ctx* ctx, double* dx) {
    if (check_ctx(ctx) || !dx) return EWG_ERR_INVALID;
    return from_split(ctx, ctx->dx, dx);
}

ewg_status ewg_apply_preconditioner(ewg_ctx* ctx, const ewg_solve_opts* o, const double* b, double* y) {
    if (check_ctx(ctx) || !o || !b || !y) return EWG_ERR_INVALID;
    cudaError_t e;
    double2 *bs = nullptr, *ys = nullptr;
    if ((e = cudaMalloc(&bs, sizeof(double2) * ctx->P.N)) != cudaSuccess) return cuda_fail(ctx, e, "alloc");
    if ((e = cudaMalloc(&ys, sizeof(double2) * ctx->P.N)) != cudaSuccess) { cudaFree(bs); return cuda_fail(ctx, e, "alloc"); }
    ewg_status st = to_split(ctx, b, bs);
    if (!st) st = solver_apply_preconditioner(ctx, o, bs, ys);
    if (!st) st = from_split(ctx, ys, y);
    cudaFree(bs);
    cudaFree(ys);
    return st;
}

ewg_status ewg_apply_jacobian(ewg_ctx* ctx, const double* x, double* y) {
    if (check_ctx(ctx) || !x || !y) return EWG_ERR_INVALID;
    cudaError_t e;
    double2 *xs = nullptr, *ys = nullptr;
    if ((e = cudaMalloc(&xs, sizeof(double2) * ctx->P.N)) != cudaSuccess) return cuda_fail(ctx, e, "alloc");
    if ((e = cudaMalloc(&ys, sizeof(double2) * ctx->P.N)) != cudaSuccess) { cudaFree(xs); return cuda_fail(ctx, e, "alloc"); }
    ewg_status st = to_split(ctx, x, xs);
    if (!st) st = solver_spmv(ctx, xs, ys);
    if (!st) st = from_split(ctx, ys, y);
    cudaFree(xs);
    cudaFree(ys);
    return st;
}

// a device pointer of this context's device with room for a 16-byte aligned double2 vector
static bool device_vector_ok(ewg_ctx* ctx, const void* p) {
    if (!p || ((uintptr_t)p & 15)) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return false;
    return a.device == ctx->device;
}

ewg_status ewg_device_buffer(ewg_ctx* ctx, int32_t which, double** out) {
    if (check_ctx(ctx) || !out) return EWG_ERR_INVALID;
    if (which == EWG_BUFFER_SOLUTION) { *out = (double*)ctx->x0; return EWG_OK; }
    if (which == EWG_BUFFER_RESIDUAL) { *out = (double*)ctx->r; return EWG_OK; }
    return EWG_ERR_INVALID;
}

ewg_status ewg_device_spmv(ewg_ctx* ctx, const double* x, double* y) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    if (!device_vector_ok(ctx, x) || !device_vector_ok(ctx, y)) { ctx->err = "device_spmv: x and y must be aligned device vectors"; return EWG_ERR_INVALID; }
    if (ctx->jacPrecision != EWG_PRECISION_FP64) { ctx->err = "device_spmv needs the FP64 Jacobian"; return EWG_ERR_INVALID; }
    return solver_spmv(ctx, (const double2*)x, (double2*)y);
}

ewg_status ewg_device_precondition(ewg_ctx* ctx, const ewg_solve_opts* o, const double* b, double* y) {
    if (check_ctx(ctx) || !o) return EWG_ERR_INVALID;
    if (!device_vector_ok(ctx, b) || !device_vector_ok(ctx, y)) { ctx->err = "device_precondition: b and y must be aligned device vectors"; return EWG_ERR_INVALID; }
    return solver_apply_preconditioner(ctx, o, (const double2*)b, (double2*)y);
}

static ewg_status slab_args_ok(ewg_ctx* ctx, std::initializer_list<const void*> vecs, const void* out, const char* what) {
    for (const void* v : vecs)
        if (!device_vector_ok(ctx, (const double*)v)) {
            ctx->err = std::string(what) + ": vectors must be aligned device vectors";
            return EWG_ERR_INVALID;
        }
    if (out && ((uintptr_t)out % sizeof(double)) != 0) {
        ctx->err = std::string(what) + ": misaligned output";
        return EWG_ERR_INVALID;
    }
    return EWG_OK;
}

static bool device_ptr_ok(ewg_ctx* ctx, const void* p) {
    if (!p || ((uintptr_t)p & 7)) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == ctx->device;
}

ewg_status ewg_device_bicg_p(ewg_ctx* ctx, double* p, const double* r, double* r0, double* v, const void* state) {
    if (check_ctx(ctx) || !device_ptr_ok(ctx, state)) return EWG_ERR_INVALID;
    ewg_status st = slab_args_ok(ctx, {p, r, r0, v}, nullptr, "device_bicg_p");
    if (st) return st;
    return solver_slab(ctx, 0, (double2*)p, (double2*)r, (double2*)r0, (double2*)v, nullptr, state, 0, 0, nullptr);
}

ewg_status ewg_device_bicg_spmv_dot(ewg_ctx* ctx, const double* x, double* y, const double* w, int64_t lo, int64_t hi,
                                    const void* state, double* out) {
    if (check_ctx(ctx) || !out || (state && !device_ptr_ok(ctx, state))) return EWG_ERR_INVALID;
    if (ctx->jacPrecision != EWG_PRECISION_FP64) { ctx->err = "device_bicg_spmv_dot needs the FP64 Jacobian"; return EWG_ERR_INVALID; }
    ewg_status st = slab_args_ok(ctx, {x, y, w}, out, "device_bicg_spmv_dot");
    if (st) return st;
    return solver_slab(ctx, 1, (double2*)x, (double2*)y, (double2*)w, nullptr, nullptr, state, lo, hi, out);
}

ewg_status ewg_device_bicg_hs(ewg_ctx* ctx, double* x, const double* y, double* r, const double* v, int64_t lo,
                              int64_t hi, const void* state, double* out) {
    if (check_ctx(ctx) || !out || !device_ptr_ok(ctx, state)) return EWG_ERR_INVALID;
    ewg_status st = slab_args_ok(ctx, {x, y, r, v}, out, "device_bicg_hs");
    if (st) return st;
    return solver_slab(ctx, 2, (double2*)x, (double2*)y, (double2*)r, (double2*)v, nullptr, state, lo, hi, out);
}

ewg_status ewg_device_bicg_spmv_dot2(ewg_ctx* ctx, const double* z, double* t, const double* s, int64_t lo, int64_t hi,
                                     const void* state, double* out) {
    if (check_ctx(ctx) || !out || (state && !device_ptr_ok(ctx, state))) return EWG_ERR_INVALID;
    if (ctx->jacPrecision != EWG_PRECISION_FP64) { ctx->err = "device_bicg_spmv_dot2 needs the FP64 Jacobian"; return EWG_ERR_INVALID; }
    ewg_status st = slab_args_ok(ctx, {z, t, s}, out, "device_bicg_spmv_dot2");
    if (st) return st;
    return solver_slab(ctx, 3, (double2*)z, (double2*)t, (double2*)s, nullptr, nullptr, state, lo, hi, out);
}

ewg_status ewg_device_bicg_xr(ewg_ctx* ctx, double* x, const double* z, double* r, const double* t, const double* r0,
                              int64_t lo, int64_t hi, const void* state, double* out) {
    if (check_ctx(ctx) || !out || !device_ptr_ok(ctx, state)) return EWG_ERR_INVALID;
    ewg_status st = slab_args_ok(ctx, {x, z, r, t, r0}, out, "device_bicg_xr");
    if (st) return st;
    return solver_slab(ctx, 4, (double2*)x, (double2*)z, (double2*)r, (double2*)t, (const double2*)r0, state, lo, hi,
                       out);
}

int32_t ewg_device_bicg_state_size(void) { return solver_slab_state_size(); }

ewg_status ewg_device_bicg_state(ewg_ctx* ctx, int32_t stage, void* state, const double* red, const ewg_solve_opts* o) {
    if (check_ctx(ctx) || !device_ptr_ok(ctx, state) || !device_ptr_ok(ctx, red)) return EWG_ERR_INVALID;
    if (stage == 0 && !o) { ctx->err = "device_bicg_state: stage 0 needs the solve options"; return EWG_ERR_INVALID; }
    return solver_slab_state(ctx, stage, state, red, o);
}

ewg_status ewg_device_bicg_state_read(ewg_ctx* ctx, const void* state, int32_t* status, int32_t* iterations,
                                      int32_t* restarts, double* res, double* init) {
    if (check_ctx(ctx) || !device_ptr_ok(ctx, state)) return EWG_ERR_INVALID;
    return solver_slab_state_read(ctx, state, status, iterations, restarts, res, init);
}

ewg_status ewg_newton_update(ewg_ctx* ctx) {
    if (check_ctx(ctx)) return EWG_ERR_INVALID;
    int bad = 0;
    ewg_status st = solver_newton_update(ctx, &bad);
    if (st) return st;
    if (bad) { ctx->err = "Non-finite update!"; return EWG_ERR_NONFINITE; }
    return EWG_OK;
}

ewg_status ewg_newton_apply(ewg_ctx* ctx, double dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                            ewg_newton_report* rep) {
    if (check_ctx(ctx) || !no || !so || !rep) return EWG_ERR_INVALID;
    memset(rep, 0, sizeof(*rep));
    ctx->jacPrecision = so->precision;
    int numIterations = 0;
    double error = 1e100, lastError = 1e100;
    auto converged = [&]() { return error <= no->newton_tolerance; };
    auto proceed = [&]() {
        if (numIterations < 1) return true;
        if (converged()) return false;
        if (numIterations >= no->newton_max_iterations) return error * 4.0 < lastError;
        return true;
    };
    // model.update() calls updateBegin() right before NewtonMethod::apply (fvbasediscretization.hh:1242)
    ewg_status status = update_reference_pressure(ctx, true);
    while (status == EWG_OK && proceed()) {
        lastError = error;
        ewg_lin_report lr = {};
        ewg_status st = linearize_impl(ctx, dt, &lr);
        rep->t_linearize += lr.seconds;
        if (st) { status = st; break; }
        lastError = error;
        error = lr.error;
        if (no->verbose) fprintf(stderr, "Newton iteration %d error: %g\n", numIterations, error);
        if (error > no->newton_max_error) { status = EWG_ERR_MAX_ERROR; ctx->err = "Newton: error above NewtonMaxError"; break; }
        if (!proceed()) { ++numIterations; break; }
        ewg_solve_report sr = {};
        st = solver_solve(ctx, so, &sr);
        rep->t_solve += sr.seconds;
        rep->linear_iterations += sr.iterations;
        if (st) { status = st; break; }
        cudaEventRecord(ctx->ev0, ctx->stream);
        int bad = 0;
        st = solver_newton_update(ctx, &bad);
        cudaEventRecord(ctx->ev1, ctx->stream);
        cudaEventSynchronize(ctx->ev1);
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        rep->t_update += ms * 1e-3;
        if (st) { status = st; break; }
        if (bad) { status = EWG_ERR_NONFINITE; ctx->err = "Non-finite update!"; break; }
        ++numIterations;
    }
    rep->iterations = numIterations;
    rep->error = error;
    if (status == EWG_OK && !converged()) { status = EWG_ERR_NOT_CONVERGED; ctx->err = "Newton did not converge"; }
    rep->converged = status == EWG_OK;
    rep->status = status;
    return status;
}

}  // extern "C"
