// Internal declarations of the B200 ECFV linearizer / BiCGStab solver (libewg.so).
//
// Device storage order ("red-black split"): cell c = i + nx*(j + ny*k) has colour
// col(c) = (i + j + k) & 1 and half index h(c) = c >> 1; it lives at s(c) = col*Nh + h with
// Nh = N/2. nx is even, so the pair {2h, 2h+1} always holds one red and one black cell of the same
// x-row, every colour holds exactly Nh cells, and a cell's face neighbours (all of the other
// colour) sit at half indices h-1+b / h+b (x), h -/+ nx/2 (y), h -/+ nx*ny/2 (z) where b is the
// cell's position in its pair. A warp of consecutive h therefore reads and writes contiguous
// 8/16-byte words in every array and every neighbour stream.
//
// Jacobian: the reference's BCRS pattern (fvbaselinearizer.hh:303-340) is, on a structured grid,
// the 5-point (2D) / 7-point (3D) block stencil, so it is stored band-major with implicit columns:
// plane (band*4 + q)[s] holds entry q = 2*eq + pv of the block of row s in band
//   0 diagonal, 1 -x, 2 +x, 3 -y, 4 +y, 5 -z, 6 +z.
// Bands of missing neighbours (boundary rows) stay zero forever.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/ewg.h"

namespace ewg {

constexpr int kMaxBands = 7;

// Regularised material law of one region with the constants RegularizedVanGenuchtenParams /
// RegularizedBrooksCoreyParams derive in finalize().
struct LawDev {
    int kind;
    double swr, snr, den;           // den = 1 - (swr + snr)
    // van Genuchten
    double alpha, n, m, negInvM, invN, invM, twoM;
    double pcLowSw, pcHighSw, pcLow, pcSlopeLow, m1High;
    double spX0, spH, spY0, spY1, spHM0, spHM1;  // Hermite segment on [x0, x0 + h]
    // Brooks-Corey
    double pe, negInvLambda, krwExp, krnExp, bcLowSw, bcPcLow, bcSlopeLow, bcSlopeOne;
};

// Division by a run-time invariant divisor d >= 1 for 0 <= n < 2^32 with one multiply-high
// (Granlund and Montgomery, "Division by invariant integers using multiplication", PLDI 1994):
// q = (t + ((n - t) >> s1)) >> s2 with t = mulhi(m, n), m = floor(2^32 (2^l - d) / d) + 1,
// l = ceil(log2 d), (s1, s2) = (1, l - 1); d = 1 uses m = 0, s1 = s2 = 0.
struct FastDiv {
    uint32_t d, m, s1, s2;
};
inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    if (d <= 1) {
        f.d = 1; f.m = 0; f.s1 = 0; f.s2 = 0;
        return f;
    }
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    f.s1 = 1;
    f.s2 = l - 1;
    return f;
}
__host__ __device__ inline uint32_t fastdiv(const FastDiv& f, uint32_t n) {
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(f.m, n);
#else
    const uint32_t t = (uint32_t)(((uint64_t)f.m * n) >> 32);
#endif
    return (t + ((n - t) >> f.s1)) >> f.s2;
}

// Everything a kernel needs about the problem, passed by value.
struct Phys {
    int dim, nx, ny, nz;
    int64_t N, Nh;
    int nxh;                 // nx / 2
    int64_t planeh;          // nx * ny / 2
    int nb;                  // number of bands: 1 + 2*dim
    double h[3], L[3];
    double vol, area[3];
    double porosity, rho[2], mu[2], g;  // gravity vector (0, -g, 0)
    double pRef, leftScale;
    double inletXlo, inletXhi, inletZlo, inletZhi, inletRate;
    double lensLo[3], lensHi[3], eps;
    LawDev law[2];           // 0 outer, 1 lens
    // free-flow boundary state S_w = 1 per region (filled on the device at context creation):
    // p_cnw and the phase mobilities k_r / mu
    double bndPc[2];
    double bndLam[2][2];
    // intensive quantities at S_w = 1 per region (p_c, dp_c, lambda_w, dlambda_w, lambda_n,
    // dlambda_n with d/dS_w), evaluated on the device by the same function at context creation
    double sat1[2][6];
    FastDiv fdNxh, fdNy;     // divisions by nx / 2 and ny in cell_of (N < 2^31)
    double rhoArea[3][2];    // rho_alpha * face area per axis (mass flux per unit velocity)
    double invVol;           // 1 / cell volume
    int kOrigin;             // global index of plane 0 (z-slab of a decomposed grid), else 0
    // box-8-colour solver order (3D grids with nx, ny, nz multiples of 4; see ewg_box8.cuh)
    int b8ok;                // 1 if the grid has that order
    int nbx, nby, nbz;       // 4x4x4 superblocks per axis
    int64_t Nb;              // N / 64: cells per group = superblocks
    FastDiv fdNbx, fdNby, fdNb;
};

// Geometry of one interior face seen from a cell, per (axis, cell index along the axis, side):
// the two-point gradient coefficient dA / |dA|^2 with dA = x_j - x_i along the axis
// (fvbasegradientcalculator.hh:194-240) and, for faces normal to gravity (y), the hydrostatic
// correction (pStat_j - pStat_i) / |dA|^2 of each phase (darcyfluxmodule.hh:216-290). The values
// are computed on the host with the same IEEE operations the kernels would use, so reading them
// from the table gives the same bits as recomputing them per cell.
struct FaceGeo {
    double coef, dA, gt[2];
};
// Index of (axis, idx, side) in the face-geometry table.
__host__ __device__ inline int face_geo_index(const int n[3], int axis, int idx, int side) {
    int off = axis == 0 ? 0 : (axis == 1 ? 2 * n[0] : 2 * (n[0] + n[1]));
    return off + 2 * idx + side;
}

// Derived index constants of the split storage order from dim, nx, ny, nz.
inline void set_index_constants(Phys& P) {
    if (P.dim == 2) P.nz = 1;
    P.N = (int64_t)P.nx * P.ny * P.nz;
    P.Nh = P.N / 2;
    P.nxh = P.nx / 2;
    P.planeh = (int64_t)P.nx * P.ny / 2;
    P.nb = 1 + 2 * P.dim;
    P.fdNxh = make_fastdiv((uint32_t)P.nxh);
    P.fdNy = make_fastdiv((uint32_t)P.ny);
    P.b8ok = P.dim == 3 && P.nx % 4 == 0 && P.ny % 4 == 0 && P.nz % 4 == 0 && P.N >= 64 ? 1 : 0;
    P.nbx = P.nx / 4;
    P.nby = P.ny / 4;
    P.nbz = P.nz / 4;
    P.Nb = P.N / 64;
    P.fdNbx = make_fastdiv((uint32_t)(P.nbx > 0 ? P.nbx : 1));
    P.fdNby = make_fastdiv((uint32_t)(P.nby > 0 ? P.nby : 1));
    P.fdNb = make_fastdiv((uint32_t)(P.Nb > 0 ? P.Nb : 1));
}

struct CellIdx {
    int64_t c;               // natural index
    int i, j, k;
    int b;                   // position inside the pair (c & 1)
};

__host__ __device__ inline CellIdx cell_of(const Phys& P, int col, int64_t h) {
    CellIdx r;
    const uint32_t hh = (uint32_t)h;
    const uint32_t row = fastdiv(P.fdNxh, hh);   // x-row index j + ny*k
    const uint32_t hx = hh - row * (uint32_t)P.nxh;
    const uint32_t k = fastdiv(P.fdNy, row);
    r.j = (int)(row - k * (uint32_t)P.ny);
    r.k = (int)k;
    r.b = col ^ ((r.j + r.k) & 1);
    r.i = (int)(2 * hx + r.b);
    r.c = (int64_t)row * P.nx + r.i;
    return r;
}

__host__ __device__ inline int64_t split_of(const Phys& P, int64_t c) {
    int i = (int)(c % P.nx);
    int64_t row = c / P.nx;
    int j = (int)(row % P.ny), k = (int)(row / P.ny);
    int col = (i + j + k) & 1;
    return col * P.Nh + (c >> 1);
}

// Band of the face in direction (axis, side): 1 + 2*axis + side.
__host__ __device__ inline int band_of(int axis, int side) { return 1 + 2 * axis + side; }
__host__ __device__ inline int opposite_band(int band) { return band == 0 ? 0 : (((band - 1) ^ 1) + 1); }

// Split-order position of the neighbour of cell (col, h, b) across face (axis, side), or -1.
__host__ __device__ inline int64_t neighbour_split(const Phys& P, int col, int64_t h, const CellIdx& ci,
                                                   int axis, int side) {
    int64_t base = (int64_t)(col ^ 1) * P.Nh;
    if (axis == 0) {
        if (side == 0) return ci.i > 0 ? base + h - 1 + ci.b : -1;
        return ci.i < P.nx - 1 ? base + h + ci.b : -1;
    }
    if (axis == 1) {
        if (side == 0) return ci.j > 0 ? base + h - P.nxh : -1;
        return ci.j < P.ny - 1 ? base + h + P.nxh : -1;
    }
    if (side == 0) return ci.k > 0 ? base + h - P.planeh : -1;
    return ci.k < P.nz - 1 ? base + h + P.planeh : -1;
}

// ---- kernel profiling ----------------------------------------------------------------------

// Kernel classes counted on every launch and, with profiling on, timed with a CUDA event pair on
// the context stream (the device-side analogue of the reference's linearize / solve / update
// timers, newtonmethod.hh:488-500).
enum KernelId {
    K_INTENSIVE = 0, K_ASSEMBLE, K_STORAGE, K_INITIAL, K_LAYOUT,
    K_DIAG_INVERSE, K_ILU_BLACK_FACTOR, K_ILU_BLACK_APPLY, K_ILU_RED_APPLY, K_JACOBI_APPLY,
    K_SPMV, K_BICG_INIT, K_BICG_P, K_BICG_SPMV_ALPHA, K_BICG_HS, K_BICG_SPMV_OMEGA, K_BICG_XR,
    K_TO_FLOAT, K_DEFECT_ACCUMULATE, K_DEFECT_RESIDUAL, K_NEWTON_UPDATE, K_BCRS,
    K_BICG_TRUE_RESIDUAL,
    K_B8_LAYOUT, K_B8_FACTOR, K_B8_FORWARD, K_B8_BACKWARD,
    K_NUM_KERNELS
};
extern const char* const kKernelNames[K_NUM_KERNELS];

struct Profiler {
    static constexpr int kPool = 1024;
    bool on = false;
    int period = 1;                     // time every period-th launch of each class
    bool pendingTimed = false;
    long long sampled[K_NUM_KERNELS] = {};
    cudaEvent_t ev[2 * kPool] = {};
    int pendId[kPool] = {};
    int npend = 0;
    bool created = false;
    double ms[K_NUM_KERNELS] = {};
    long long launches[K_NUM_KERNELS] = {};
};

}  // namespace ewg

struct ewg_ctx {
    ewg::Phys P;
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    int jacPrecision = EWG_PRECISION_FP64;   // what ewg_linearize writes
    int localLinearizer = EWG_LOCAL_LINEARIZER_AD;  // LocalLinearizerSplice
    int fdMethod = 1;                        // NumericDifferenceMethod of the FD linearizer
    double refPressure = -1.0;               // ImmiscibleModel::updateBegin's reference pressure (unset)
    bool jacFromLinearizer = false;          // J/r valid
    bool iluValid = false;
    int iluKind = -1, iluPrecision = -1, iluOrder = -1;
    // host copy of the reference BCRS pattern
    int64_t nnzb = 0;
    int32_t* d_rowPtr = nullptr;             // device BCRS pattern (for export / import)
    int32_t* d_colIdx = nullptr;
    // state (split order)
    double2* x0 = nullptr;      // solution(0)
    double2* x1 = nullptr;      // solution(1)
    double2* sold = nullptr;    // storage of solution(1) per unit volume
    double* perm = nullptr;
    uint8_t* lens = nullptr;
    double* iq = nullptr;       // 6 planes: pc, dpc, lw, dlw, ln, dln
    ewg::FaceGeo* geo = nullptr;     // face-geometry table (3D fast path)
    double2* r = nullptr;       // residual
    double* J = nullptr;        // nb*4 planes, FP64
    float* J32 = nullptr;       // nb*4 planes, FP32 (mixed precision)
    unsigned long long* d_errmax = nullptr;  // max|r| as ordered bits
    int* d_flags = nullptr;                  // [0] nonfinite
    // solver
    double2* dx = nullptr;      // solution update
    double2* d_stage = nullptr; // natural-order staging for host transfers
    void* sv = nullptr;         // solver workspace (vectors, ILU factors), owned by the solver
    size_t svBytes = 0;
    // host staging
    double* h_pinned = nullptr;
    size_t h_pinnedBytes = 0;
    // bytes copied between the caller's host buffers and the device by the entry points
    // (ewg_transfer_counters); the library's own control reads are not counted
    uint64_t h2dBytes = 0, d2hBytes = 0;
    ewg::Profiler prof;
};

namespace ewg {

// ---- host helpers implemented across the .cu files --------------------------------------
void prof_begin(ewg_ctx* ctx, int id);
void prof_end(ewg_ctx* ctx, int id);
void prof_flush(ewg_ctx* ctx);  // call after the stream is synchronised

// Launch a kernel on the context stream, counted and (with profiling on) timed.
#define EWG_LAUNCH(ctx, id, kernel, grid, block, ...)                      \
    do {                                                                 \
        ::ewg::prof_begin((ctx), (id));                                  \
        kernel<<<(grid), (block), 0, (ctx)->stream>>>(__VA_ARGS__);      \
        ::ewg::prof_end((ctx), (id));                                    \
    } while (0)

// Launch with programmatic stream serialization (the kernel must start with pdl_enter): the
// kernel's launch and block setup overlap the end of the previous kernel in the stream. EWG_PDL=0
// at compile time launches these kernels like EWG_LAUNCH.
#ifndef EWG_PDL
#define EWG_PDL 1
#endif
template <typename... KArgs, typename... Args>
inline void launch_pdl(cudaStream_t stream, void (*kernel)(KArgs...), int grid, int block, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = EWG_PDL;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}
#define EWG_LAUNCH_PDL(ctx, id, kernel, grid, block, ...)                          \
    do {                                                                         \
        ::ewg::prof_begin((ctx), (id));                                          \
        ::ewg::launch_pdl((ctx)->stream, kernel, (grid), (block), __VA_ARGS__);  \
        ::ewg::prof_end((ctx), (id));                                            \
    } while (0)

void build_phys(Phys& P, const ewg_grid* g, const ewg_problem* p);
ewg_status cuda_fail(ewg_ctx* ctx, cudaError_t e, const char* what);
int grid_size_for(ewg_ctx* ctx, const void* kernel, int block, size_t smem = 0);

// linearization (ewg_linearize.cu)
ewg_status launch_storage(ewg_ctx* ctx, const double2* x, double2* sold);
ewg_status launch_linearize(ewg_ctx* ctx, double dt, bool withJacobian, const double2* x,
                            double2* r, double* maxOut, int* nonfinite);
ewg_status launch_initial_solution(ewg_ctx* ctx, double2* x);
// intensive quantities (p_c, lambda_w, lambda_n with d/dS_w) of state x into ctx->iq
ewg_status launch_intensive(ewg_ctx* ctx, const double2* x);
ewg_status compute_boundary_constants(ewg_ctx* ctx);
// face-geometry table of a 3D grid (allocated on the device)
ewg_status build_interior_tables(ewg_ctx* ctx);
// host side of the same: 2 (nx + ny + nz) entries in face_geo_index order
void build_face_geo(const Phys& P, std::vector<FaceGeo>& geo);
// the S_w = 1 free-flow boundary constants of P (bndPc, bndLam), computed on the device
cudaError_t boundary_constants(Phys& P, cudaStream_t stream);
// layout kernels for problems without a context (ensemble members)
cudaError_t layout_natural_to_split(const Phys& P, cudaStream_t st, const double2* nat, double2* spl);
cudaError_t layout_split_to_natural(const Phys& P, cudaStream_t st, const double2* spl, double2* nat);
cudaError_t layout_scalar_to_split(const Phys& P, cudaStream_t st, const double* nat, double* spl);
cudaError_t layout_lens_flags(const Phys& P, cudaStream_t st, uint8_t* lens);

// solver (ewg_solver.cu)
ewg_status solver_solve(ewg_ctx* ctx, const ewg_solve_opts* o, ewg_solve_report* rep);
ewg_status solver_apply_preconditioner(ewg_ctx* ctx, const ewg_solve_opts* o, const double2* b,
                                       double2* y);
ewg_status solver_spmv(ewg_ctx* ctx, const double2* x, double2* y);
ewg_status solver_slab(ewg_ctx* ctx, int kind, double2* a, double2* b, double2* c, double2* d, const double2* e,
                       const void* state, int64_t lo, int64_t hi, double* out);
ewg_status solver_slab_state(ewg_ctx* ctx, int stage, void* state, const double* red, const ewg_solve_opts* o);
int32_t solver_slab_state_size();
ewg_status solver_slab_state_read(ewg_ctx* ctx, const void* state, int32_t* status, int32_t* iterations,
                                  int32_t* restarts, double* res, double* init);
ewg_status solver_newton_update(ewg_ctx* ctx, int* nonfinite);
void solver_free(ewg_ctx* ctx);

// layout conversion (ewg_api.cu)
ewg_status to_split(ewg_ctx* ctx, const double* host_natural, double2* dev_split);
ewg_status from_split(ewg_ctx* ctx, const double2* dev_split, double* host_natural);

}  // namespace ewg
