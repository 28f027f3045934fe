// Learned Newton initial guess: a 4-layer 3D convolutional network (3x3x3 kernels, channels
// 5 -> 32 -> 32 -> 32 -> 2, ReLU between layers) that maps the state at the start of an implicit
// step (p_w, S_n, ln K, porosity, dt) to the step's increment (dp_w, dS_n). It has no reference
// counterpart; it plugs into the hook where the reference copies solution(1) into solution(0)
// (fvbasediscretization.hh:1396-1407, updateBegin :1311) and keeps the previous-step guess as the
// fallback when the predicted guess has the larger initial residual.
//
// Numerics: BF16 weights, activations and activation gradients; FP32 accumulation, FP32 master
// weights and Adam moments. Layout: channels-last, one volume after another (natural cell order
// x fastest), Cin padded to 16 or 32, the last layer's 2 outputs padded to 8 (16 for gradients).
//
// Kernels
//   k_conv3d_tc    implicit-GEMM convolution on the 5th-generation tensor cores (tcgen05.mma
//                  BF16 -> FP32 in tensor memory, TMA loads of the shifted input boxes; see
//                  ewg_conv_tc.cuh): the three 32-channel layers of the forward pass (bias, ReLU)
//                  and the three input-gradient convolutions (flipped, transposed weights;
//                  epilogue multiplies by the ReLU mask of the layer below).
//   k_conv3d       warp-level implicit-GEMM convolution (mma.sync m16n8k16 BF16 -> FP32): one
//                  warp computes 16 voxels x Cout; K = 27 taps x Cin. The 2-output last layer.
//   k_conv3d_wgrad weight and bias gradients on FP32 CUDA cores, one block per (tap, voxel chunk).
//   k_adam         Adam update of the FP32 master weights, then BF16 working copies.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "ewg_internal.cuh"
#include "ewg_conv_tc.cuh"

namespace ewg {

constexpr int kNetLayers = 4;
constexpr int kCin[kNetLayers] = {16, 32, 32, 32};   // padded input channels
constexpr int kCout[kNetLayers] = {32, 32, 32, 8};   // padded output channels
constexpr int kCinReal[kNetLayers] = {5, 32, 32, 32};
constexpr int kCoutReal[kNetLayers] = {32, 32, 32, 2};
constexpr int kTaps = 27;

struct VolDims {
    int D, H, W;   // z, y, x extents of every volume in the batch
    int B;         // volumes
    __host__ __device__ int64_t V() const { return (int64_t)B * D * H * W; }
};

// ---- tensor-core convolution --------------------------------------------------------------

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// neighbour voxel of v across tap (dz, dy, dx) in {-1,0,1}^3, or -1 outside the volume (zero padding)
__device__ __forceinline__ int64_t tap_neighbour(const VolDims& d, int64_t v, int tap) {
    if (v < 0) return -1;
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
    const int64_t per = (int64_t)d.D * d.H * d.W;
    const int64_t b = v / per;
    int64_t r = v - b * per;
    const int x = (int)(r % d.W);
    r /= d.W;
    const int y = (int)(r % d.H);
    const int z = (int)(r / d.H);
    const int nx = x + dx, ny = y + dy, nz = z + dz;
    if (nx < 0 || nx >= d.W || ny < 0 || ny >= d.H || nz < 0 || nz >= d.D) return -1;
    return b * per + ((int64_t)nz * d.H + ny) * d.W + nx;
}

// epilogue modes
constexpr int EPI_BIAS_RELU = 0;   // y = relu(acc + bias)       (BF16 out)
constexpr int EPI_BIAS = 1;        // y = acc + bias             (FP32 out, the last layer)
constexpr int EPI_MASK = 2;        // y = acc * (mask > 0)       (BF16 out, input gradients)

// One warp: 16 voxels (rows) x COUT channels. W is [27][COUT][CIN] BF16 in shared memory.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(128) k_conv3d(VolDims d, const __nv_bfloat16* __restrict__ in,
                                                 const __nv_bfloat16* __restrict__ Wg,
                                                 const float* __restrict__ bias,
                                                 const __nv_bfloat16* __restrict__ mask, int maskC,
                                                 void* __restrict__ outp, int outC) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(smem);
    const int nW = kTaps * COUT * CIN;
    for (int t = threadIdx.x; t < nW / 8; t += blockDim.x)
        reinterpret_cast<uint4*>(Ws)[t] = reinterpret_cast<const uint4*>(Wg)[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int64_t V = d.V();
    const int64_t tiles = (V + 15) / 16;
    constexpr int NT = COUT / 8;
    for (int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp; tile < tiles;
         tile += (int64_t)gridDim.x * (blockDim.x >> 5)) {
        const int64_t v0 = tile * 16 + g, v1 = v0 + 8;
        const int64_t r0 = v0 < V ? v0 : -1, r1 = v1 < V ? v1 : -1;
        float acc[NT][4];
#pragma unroll
        for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
        for (int tap = 0; tap < kTaps; ++tap) {
            const int64_t a = tap_neighbour(d, r0, tap), b = tap_neighbour(d, r1, tap);
            const uint32_t* pa = a >= 0 ? reinterpret_cast<const uint32_t*>(in + a * CIN) : nullptr;
            const uint32_t* pb = b >= 0 ? reinterpret_cast<const uint32_t*>(in + b * CIN) : nullptr;
#pragma unroll
            for (int c0 = 0; c0 < CIN; c0 += 16) {
                uint32_t A[4];
                const int k = (c0 >> 1) + q;  // 32-bit word index of channel pair c0 + 2q
                A[0] = pa ? __ldg(pa + k) : 0u;
                A[1] = pb ? __ldg(pb + k) : 0u;
                A[2] = pa ? __ldg(pa + k + 4) : 0u;
                A[3] = pb ? __ldg(pb + k + 4) : 0u;
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    const uint32_t* wrow = reinterpret_cast<const uint32_t*>(Ws + ((size_t)tap * COUT + n * 8 + g) * CIN);
                    uint32_t Bf[2] = {wrow[k], wrow[k + 4]};
                    mma_bf16(acc[n], A, Bf);
                }
            }
        }
        // epilogue: rows v0 (acc[.][0..1]) and v1 (acc[.][2..3]), columns n*8 + 2q + {0,1}
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            const int c = n * 8 + 2 * q;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t v = h ? v1 : v0;
                if (v >= V) continue;
                float y0 = acc[n][2 * h], y1 = acc[n][2 * h + 1];
                if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS) { y0 += bias[c]; y1 += bias[c + 1]; }
                if (EPI == EPI_BIAS_RELU) { y0 = fmaxf(y0, 0.f); y1 = fmaxf(y1, 0.f); }
                if (EPI == EPI_MASK) {
                    const __nv_bfloat16* m = mask + v * maskC + c;
                    if (!(__bfloat162float(m[0]) > 0.f)) y0 = 0.f;
                    if (!(__bfloat162float(m[1]) > 0.f)) y1 = 0.f;
                }
                if (EPI == EPI_BIAS) {
                    float* o = reinterpret_cast<float*>(outp) + v * outC + c;
                    if (c < outC) o[0] = y0;
                    if (c + 1 < outC) o[1] = y1;
                } else {
                    __nv_bfloat162 p = __floats2bfloat162_rn(y0, y1);
                    *reinterpret_cast<__nv_bfloat162*>(reinterpret_cast<__nv_bfloat16*>(outp) + v * outC + c) = p;
                }
            }
        }
    }
}

// dW[tap][co][ci] += sum_v dY[v][co] X[nbr(v, tap)][ci], db[co] += sum_v dY[v][co]; FP32 atomics
// per block after a block-local accumulation over a chunk of voxels. blockDim = COUT * CIN / 4.
template <int CIN, int COUT>
__global__ void k_conv3d_wgrad(VolDims d, const __nv_bfloat16* __restrict__ X, const __nv_bfloat16* __restrict__ dY,
                               int dyC, float* __restrict__ dW, float* __restrict__ db, int64_t chunk) {
    const int tap = blockIdx.y;
    const int co = threadIdx.x / (CIN / 4), ci = (threadIdx.x % (CIN / 4)) * 4;
    const int64_t V = d.V();
    const int64_t vb = (int64_t)blockIdx.x * chunk, ve = vb + chunk < V ? vb + chunk : V;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, ab = 0.f;
    for (int64_t v = vb; v < ve; ++v) {
        const float g = __bfloat162float(dY[v * dyC + co]);
        if (tap == 13) ab += g;
        const int64_t nb = tap_neighbour(d, v, tap);
        if (nb < 0 || g == 0.f) continue;
        const __nv_bfloat162* xp = reinterpret_cast<const __nv_bfloat162*>(X + nb * CIN + ci);
        const float2 x01 = __bfloat1622float2(xp[0]), x23 = __bfloat1622float2(xp[1]);
        a0 += g * x01.x; a1 += g * x01.y; a2 += g * x23.x; a3 += g * x23.y;
    }
    float* w = dW + ((size_t)tap * COUT + co) * CIN + ci;
    atomicAdd(w, a0); atomicAdd(w + 1, a1); atomicAdd(w + 2, a2); atomicAdd(w + 3, a3);
    if (tap == 13 && ci == 0) atomicAdd(db + co, ab);
}

// ---- features, loss, optimiser ------------------------------------------------------------

struct FeatureScales {
    double pScale, lnKMean, lnKScale, phiMean, phiScale, dtScale;
};

// natural-order features of the state in split order: (p_w - p_hydrostatic)/pScale, S_n,
// (ln K - mean)/scale, (phi - mean)/scale, dt/dtScale; channels 5..15 zero
__global__ void k_features(const __grid_constant__ Phys P, const double2* __restrict__ x, const double* __restrict__ perm,
                           double dt, FeatureScales fs, __nv_bfloat16* __restrict__ out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = split_of(P, c);
        const double2 xs = x[s];
        const int j = (int)((c / P.nx) % P.ny);
        const double y = (j + 0.5) * P.h[1];
        const double phydro = P.pRef + P.rho[0] * P.g * (P.L[1] - y);
        float f[16];
        f[0] = (float)((xs.x - phydro) / fs.pScale);
        f[1] = (float)(1.0 - xs.y);
        f[2] = (float)((log(perm[s]) - fs.lnKMean) / fs.lnKScale);
        f[3] = (float)((P.porosity - fs.phiMean) / fs.phiScale);
        f[4] = (float)(dt / fs.dtScale);
        for (int k = 5; k < 16; ++k) f[k] = 0.f;
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + c * 16);
        for (int k = 0; k < 8; ++k) o[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
    }
}

// normalised target of a recorded step: ((p1 - p0)/tp, (Sn1 - Sn0)/ts) in natural order
__global__ void k_targets(const __grid_constant__ Phys P, const double2* __restrict__ x0, const double2* __restrict__ x1,
                          double tp, double ts, float* __restrict__ out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = split_of(P, c);
        const double2 a = x0[s], b = x1[s];
        out[2 * c] = (float)((b.x - a.x) / tp);
        out[2 * c + 1] = (float)(((1.0 - b.y) - (1.0 - a.y)) / ts);
    }
}

// x_guess = x_prev + de-normalised prediction. The saturation increment is applied where it
// exceeds snThreshold (S_n kept in [0, 1]); the pressure increment only with applyPressure: a
// local network's pressure error raises the residual of the stiff pressure equation, while the
// saturation near the front is what costs Newton iterations.
__global__ void k_apply_guess(const __grid_constant__ Phys P, const double2* __restrict__ xprev, const float* __restrict__ pred,
                              double tp, double ts, int applyPressure, double snThreshold, double2* __restrict__ xguess) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < P.N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = split_of(P, c);
        const double2 a = xprev[s];
        double dsn = (double)pred[2 * c + 1] * ts;
        if (fabs(dsn) < snThreshold) dsn = 0.0;
        const double sn = fmin(fmax((1.0 - a.y) + dsn, 0.0), 1.0);
        const double dp = applyPressure ? (double)pred[2 * c] * tp : 0.0;
        xguess[s] = make_double2(a.x + dp, 1.0 - sn);
    }
}

// Weighted MSE over the two outputs, sum_v (w0 e0^2 + w1 e1^2) / (2 V); gradient into channels
// 0..1 of dY (16 wide, BF16)
// Cells of the plume and its front (S_n of the input above 1e-3, or a saturation target above
// 0.05 in normalised units) weigh wFront times more: elsewhere the saturation increment is zero.
__global__ void k_mse(int64_t V, const float* __restrict__ y, const float* __restrict__ t, __nv_bfloat16* __restrict__ dY,
                      float* __restrict__ loss, float w0, float w1, const __nv_bfloat16* __restrict__ feat, float wFront) {
    float l = 0.f;
    const float inv = 1.f / (float)(2 * V);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < V; v += (int64_t)gridDim.x * blockDim.x) {
        const float e0 = y[2 * v] - t[2 * v], e1 = y[2 * v + 1] - t[2 * v + 1];
        const bool front = __bfloat162float(feat[v * 16 + 1]) > 1e-3f || fabsf(t[2 * v + 1]) > 0.05f;
        const float wf = front ? wFront : 1.f;
        l += wf * (w0 * e0 * e0 + w1 * e1 * e1);
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(dY + v * 16);
        o[0] = __floats2bfloat162_rn(2.f * wf * w0 * e0 * inv, 2.f * wf * w1 * e1 * inv);
        for (int k = 1; k < 8; ++k) o[k] = __floats2bfloat162_rn(0.f, 0.f);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l * inv);
}

__global__ void k_adam(int64_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// working copies: forward weights [tap][co][ci] and input-gradient weights
// Wt[tap'][ci][co] = W[26 - tap][co][ci] (Cin / Cout swapped, taps mirrored), both BF16
__global__ void k_cast_weights(int cin, int cout, int cinT, const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                               __nv_bfloat16* __restrict__ wt) {
    const int n = kTaps * cout * cin;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ci = i % cin, co = (i / cin) % cout, tap = i / (cin * cout);
        const __nv_bfloat16 b = __float2bfloat16(w[i]);
        wf[i] = b;
        if (wt) wt[((size_t)(26 - tap) * cin + ci) * cinT + co] = b;
    }
}

}  // namespace ewg

// ---- host object ----------------------------------------------------------------------------

using namespace ewg;

struct ewg_net {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // FP32 master parameters: per layer W [27][Cout][Cin] then b [Cout] (padded shapes)
    float* params = nullptr;
    float* grads = nullptr;
    float* adamM = nullptr;
    float* adamV = nullptr;
    int64_t nParams = 0;
    int64_t wOff[kNetLayers], bOff[kNetLayers];
    __nv_bfloat16* wf[kNetLayers] = {};   // forward weights
    __nv_bfloat16* wt[kNetLayers] = {};   // input-gradient weights (layers 1..3)
    int adamStep = 0;
    // activations of the last forward pass
    __nv_bfloat16* act[kNetLayers] = {};  // inputs of each layer: X (16), H1, H2, H3 (32)
    float* out = nullptr;                 // [V][2]
    __nv_bfloat16* grad16 = nullptr;      // dY of the last layer [V][16]
    __nv_bfloat16* gradA = nullptr;       // [V][32]
    __nv_bfloat16* gradB = nullptr;       // [V][32]
    float* target = nullptr;              // [V][2]
    float* dLoss = nullptr;
    int64_t capV = 0;
    FeatureScales fs{1e4, std::log(9.05e-12), 2.0, 0.4, 0.1, 250.0};
    double tp = 100.0, ts = 0.01;         // output scales (Pa, saturation)
    float lossW[2] = {1.f, 1.f};          // loss weights of the two outputs
    float wFront = 1.f;                   // extra loss weight of plume / front cells
    int applyPressure = 0;                // guess mode: apply the predicted pressure increment
    double snThreshold = 0.0;             // guess mode: ignore |dS_n| below this
    // recorded training samples (features BF16 [V][16], targets FP32 [V][2]) per volume
    struct Sample { __nv_bfloat16* f; float* t; int D, H, W; };
    std::vector<Sample> samples;
};

namespace {

ewg_status net_fail(ewg_net* n, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EWG_OK;
    n->err = std::string(what) + ": " + cudaGetErrorString(e);
    return EWG_ERR_CUDA;
}

int64_t layer_w(int l) { return (int64_t)kTaps * kCout[l] * kCin[l]; }

ewg_status ensure_capacity(ewg_net* n, int64_t V) {
    if (V <= n->capV) return EWG_OK;
    void* ps[] = {n->act[0], n->act[1], n->act[2], n->act[3], n->out, n->grad16, n->gradA, n->gradB, n->target};
    for (void* p : ps) if (p) cudaFree(p);
    cudaError_t e = cudaSuccess;
    if (!e) e = cudaMalloc(&n->act[0], sizeof(__nv_bfloat16) * V * 16);
    for (int l = 1; l < kNetLayers && !e; ++l) e = cudaMalloc(&n->act[l], sizeof(__nv_bfloat16) * V * 32);
    if (!e) e = cudaMalloc(&n->out, sizeof(float) * V * 2);
    if (!e) e = cudaMalloc(&n->grad16, sizeof(__nv_bfloat16) * V * 16);
    if (!e) e = cudaMalloc(&n->gradA, sizeof(__nv_bfloat16) * V * 32);
    if (!e) e = cudaMalloc(&n->gradB, sizeof(__nv_bfloat16) * V * 32);
    if (!e) e = cudaMalloc(&n->target, sizeof(float) * V * 2);
    if (e) return net_fail(n, e, "net activations");
    n->capV = V;
    return EWG_OK;
}

// ---- tensor-core convolution: tensor maps and launches ----------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver the runtime uses (no link against libcuda)
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
        cudaGetLastError();
    });
    return fn;
}

// channels-last activations [B][D][H][W][C] as the 5-D map (C, x, y, z, volume), box (C, 32, 4, 1, 1)
bool tc_map_activations(CUtensorMap* m, const __nv_bfloat16* p, int C, const VolDims& d) {
    EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t row = (cuuint64_t)C * 2;
    const cuuint64_t dims[5] = {(cuuint64_t)C, (cuuint64_t)d.W, (cuuint64_t)d.H, (cuuint64_t)d.D, (cuuint64_t)d.B};
    const cuuint64_t strides[4] = {row, row * d.W, row * d.W * d.H, row * d.W * d.H * d.D};
    const cuuint32_t box[5] = {(cuuint32_t)C, (cuuint32_t)kTcTileX, (cuuint32_t)kTcTileY, 1, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(p), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, C == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the same activations for the ring of input rows: box (8, 130, 1, 1, 1), 8 channels x 130
// x-positions of one row, no swizzle
bool tc_map_activation_lines(CUtensorMap* m, const __nv_bfloat16* p, int C, const VolDims& d) {
    EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t row = (cuuint64_t)C * 2;
    const cuuint64_t dims[5] = {(cuuint64_t)C, (cuuint64_t)d.W, (cuuint64_t)d.H, (cuuint64_t)d.D, (cuuint64_t)d.B};
    const cuuint64_t strides[4] = {row, row * d.W, row * d.W * d.H, row * d.W * d.H * d.D};
    const cuuint32_t box[5] = {8, (cuuint32_t)kTcRowX, 1, 1, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(p), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// weights [27][COUT][CIN] as the 2-D map (CIN, 27 COUT), box (CIN, COUT): one tap per box
bool tc_map_weights(CUtensorMap* m, const __nv_bfloat16* p, int cin, int cout) {
    EncodeTiledFn f = encode_tiled();
    if (!f) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cin, (cuuint64_t)kTaps * cout};
    const cuuint64_t strides[1] = {(cuuint64_t)cin * 2};
    const cuuint32_t box[2] = {(cuuint32_t)cin, (cuuint32_t)cout};
    const cuuint32_t es[2] = {1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(p), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, cin == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the device word the tensor-core convolution records a failed wait in (0: none)
static __device__ int g_convTcErr;

int* conv_tc_err_ptr() {
    int* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_convTcErr) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

// the dynamic shared-memory limit of both tilings and the largest shared-memory carveout, so that
// two CTAs (their 55 KB of weights and the TMA ring each) share an SM
template <int CIN, int COUT, int EPI>
cudaError_t conv_tc_attr() {
    cudaError_t e = cudaFuncSetAttribute(k_conv3d_tc<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         TcShape<CIN, COUT>::smemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv3d_tc<CIN, COUT, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv3d_tc_ring<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TcRingShape<CIN, COUT>::smemBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_conv3d_tc_ring<CIN, COUT, EPI>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return e;
}

// CTAs of a tensor-core convolution that fit on one SM: by shared memory (the SM's shared memory
// over the CTA's dynamic size plus the per-block reservation) and by registers (64 K in four
// sub-partitions of 16 K, a CTA's six warps spread two per sub-partition at most), at most 4.
// (cudaOccupancyMaxActiveBlocksPerMultiprocessor reports 1 for these kernels although the profiler
// shows two resident.)
int tc_resident(const void* k, int smem) {
    cudaFuncAttributes fa;
    int dev = 0, smemSM = 0, resv = 0;
    if (cudaFuncGetAttributes(&fa, k) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smemSM, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const int bySmem = smemSM / (smem + resv);
    const int regs = (fa.numRegs + 7) / 8 * 8;
    const int warpsPerSubpartition = 16384 / (regs * 32);
    const int byRegs = warpsPerSubpartition / ((kTcThreads / 32 + 3) / 4);
    int n = bySmem < byRegs ? bySmem : byRegs;
    if (n > 4) n = 4;
    return n < 1 ? 1 : n;
}

cudaError_t conv_tc_attrs() {
    cudaError_t e = conv_tc_attr<16, 32, EPI_BIAS_RELU>();
    if (!e) e = conv_tc_attr<32, 32, EPI_BIAS_RELU>();
    if (!e) e = conv_tc_attr<16, 32, EPI_MASK>();
    if (!e) e = conv_tc_attr<32, 32, EPI_MASK>();
    return e;
}

// One 3x3x3 convolution (CIN -> COUT = 32, epilogue bias + ReLU or ReLU mask) on the tensor cores:
// row tiles (one input box per z-tap feeds nine taps) for volumes at least kTcRowMinW wide, 32 x 4
// patches otherwise; false when a tensor map cannot be built.
template <int CIN, int COUT, int EPI>
bool launch_conv_tc(cudaStream_t st, const VolDims& d, const __nv_bfloat16* in, const __nv_bfloat16* W,
                    const float* bias, const __nv_bfloat16* mask, int maskC, __nv_bfloat16* out, int outC) {
    static_assert(EPI == EPI_BIAS_RELU || EPI == EPI_MASK, "tensor-core epilogues");
    CUtensorMap mi, mw;
    int* err = conv_tc_err_ptr();
    const bool rows = d.W >= kTcRowMinW;
    if (!err || !tc_map_weights(&mw, W, CIN, COUT)) return false;
    if (!(rows ? tc_map_activation_lines(&mi, in, CIN, d) : tc_map_activations(&mi, in, CIN, d))) return false;
    static int sms = 0, perSM = 0, perSMRing = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        perSM = tc_resident((const void*)k_conv3d_tc<CIN, COUT, EPI>, TcShape<CIN, COUT>::smemBytes);
        perSMRing = tc_resident((const void*)k_conv3d_tc_ring<CIN, COUT, EPI>, TcRingShape<CIN, COUT>::smemBytes);
    }
    if (rows) {
        // row tiles of 128 voxels in segments of kTcSegRows rows, input rows reused through a ring
        const int64_t nSegs = (int64_t)d.B * d.D * ((d.H + kTcSegRows - 1) / kTcSegRows) *
                              ((d.W + kTcRows - 1) / kTcRows);
        const int64_t full = (int64_t)sms * perSMRing;
        const int grid = (int)(nSegs < full ? nSegs : full);
        k_conv3d_tc_ring<CIN, COUT, EPI><<<grid, kTcThreads, TcRingShape<CIN, COUT>::smemBytes, st>>>(
            mi, mw, d.D, d.H, d.W, nSegs, bias, mask, maskC, out, outC, err);
    } else {
        // 32 x 4 patches of one z-plane
        const int64_t nTiles =
            (int64_t)d.B * d.D * ((d.H + kTcTileY - 1) / kTcTileY) * ((d.W + kTcTileX - 1) / kTcTileX);
        const int64_t full = (int64_t)sms * perSM;
        const int grid = (int)(nTiles < full ? nTiles : full);
        k_conv3d_tc<CIN, COUT, EPI><<<grid, kTcThreads, TcShape<CIN, COUT>::smemBytes, st>>>(
            mi, mw, d.D, d.H, d.W, nTiles, bias, mask, maskC, out, outC, err);
    }
    return true;
}

// After a synchronization: EWG_ERR_TIMEOUT if a tensor-core convolution gave up a wait since the
// last check (the word is cleared).
ewg_status conv_tc_check(std::string* errText) {
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_convTcErr, sizeof(int));
    if (e != cudaSuccess) {
        if (errText) *errText = std::string("read convolution status: ") + cudaGetErrorString(e);
        return EWG_ERR_CUDA;
    }
    if (v == 0) return EWG_OK;
    const int zero = 0;
    cudaMemcpyToSymbol(g_convTcErr, &zero, sizeof(int));
    if (errText) *errText = "tensor-core convolution: a bounded wait gave up (stage " + std::to_string(v) + ")";
    return EWG_ERR_TIMEOUT;
}

// The dynamic shared-memory limit of one k_conv3d instance (its weights, up to 55,296 B, are above
// the 48 KB default). The attribute belongs to the current device, so ewg_net_create sets it for
// the device the net lives on.
template <int CIN, int COUT, int EPI>
cudaError_t conv_smem_attr() {
    return cudaFuncSetAttribute(k_conv3d<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(__nv_bfloat16) * kTaps * COUT * CIN));
}

cudaError_t conv_smem_attrs() {
    cudaError_t e = conv_smem_attr<16, 32, EPI_BIAS_RELU>();
    if (!e) e = conv_smem_attr<32, 32, EPI_BIAS_RELU>();
    if (!e) e = conv_smem_attr<32, 8, EPI_BIAS>();
    if (!e) e = conv_smem_attr<16, 32, EPI_MASK>();
    if (!e) e = conv_smem_attr<32, 32, EPI_MASK>();
    if (!e) e = conv_tc_attrs();
    return e;
}

template <int CIN, int COUT, int EPI>
void launch_conv(ewg_net* n, const VolDims& d, const __nv_bfloat16* in, const __nv_bfloat16* W, const float* bias,
                 const __nv_bfloat16* mask, int maskC, void* out, int outC) {
    const size_t smem = sizeof(__nv_bfloat16) * kTaps * COUT * CIN;
    auto k = k_conv3d<CIN, COUT, EPI>;
    const int64_t tiles = (d.V() + 15) / 16;
    int64_t blocks = (tiles + 3) / 4;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k<<<(int)blocks, 128, smem, n->stream>>>(d, in, W, bias, mask, maskC, out, outC);
}

// forward pass over the features already in act[0]: the three 32-channel layers on the
// tensor cores (tcgen05), the 2-output layer with the warp-level kernel
ewg_status forward(ewg_net* n, const VolDims& d) {
    const float* p = n->params;
    bool ok = launch_conv_tc<16, 32, EPI_BIAS_RELU>(n->stream, d, n->act[0], n->wf[0], p + n->bOff[0], nullptr, 0,
                                                    n->act[1], 32);
    ok = ok && launch_conv_tc<32, 32, EPI_BIAS_RELU>(n->stream, d, n->act[1], n->wf[1], p + n->bOff[1], nullptr, 0,
                                                     n->act[2], 32);
    ok = ok && launch_conv_tc<32, 32, EPI_BIAS_RELU>(n->stream, d, n->act[2], n->wf[2], p + n->bOff[2], nullptr, 0,
                                                     n->act[3], 32);
    if (!ok) {
        n->err = "tensor map of a convolution could not be built";
        return EWG_ERR_CUDA;
    }
    launch_conv<32, 8, EPI_BIAS>(n, d, n->act[3], n->wf[3], p + n->bOff[3], nullptr, 0, n->out, 2);
    return EWG_OK;
}

template <int CIN, int COUT>
void launch_wgrad(ewg_net* n, const VolDims& d, const __nv_bfloat16* X, const __nv_bfloat16* dY, int dyC, int l) {
    const int64_t chunk = 512;
    const int64_t nb = (d.V() + chunk - 1) / chunk;
    dim3 grid((unsigned)nb, kTaps);
    k_conv3d_wgrad<CIN, COUT><<<grid, COUT * CIN / 4, 0, n->stream>>>(d, X, dY, dyC, n->grads + n->wOff[l],
                                                                        n->grads + n->bOff[l], chunk);
}

// backward pass after forward(); dY of the last layer in grad16; gradients accumulate in grads.
// The input gradients are convolutions with the flipped, transposed weights on the tensor cores.
ewg_status backward(ewg_net* n, const VolDims& d) {
    // layer 4: X = H3 (32), dY (16 wide, 8 used)
    launch_wgrad<32, 8>(n, d, n->act[3], n->grad16, 16, 3);
    // dH3 = conv(dY, W4t) * (H3 > 0): Cin' = 16 (8 real + 8 zero), Cout' = 32
    bool ok = launch_conv_tc<16, 32, EPI_MASK>(n->stream, d, n->grad16, n->wt[3], nullptr, n->act[3], 32, n->gradA, 32);
    launch_wgrad<32, 32>(n, d, n->act[2], n->gradA, 32, 2);
    ok = ok && launch_conv_tc<32, 32, EPI_MASK>(n->stream, d, n->gradA, n->wt[2], nullptr, n->act[2], 32, n->gradB, 32);
    launch_wgrad<32, 32>(n, d, n->act[1], n->gradB, 32, 1);
    ok = ok && launch_conv_tc<32, 32, EPI_MASK>(n->stream, d, n->gradB, n->wt[1], nullptr, n->act[1], 32, n->gradA, 32);
    launch_wgrad<16, 32>(n, d, n->act[0], n->gradA, 32, 0);
    if (!ok) {
        n->err = "tensor map of a convolution could not be built";
        return EWG_ERR_CUDA;
    }
    return EWG_OK;
}

ewg_status refresh_weights(ewg_net* n) {
    for (int l = 0; l < kNetLayers; ++l) {
        const int cinT = kCout[l] == 8 ? 16 : kCout[l];  // the gradient layout of the last layer is 16 wide
        k_cast_weights<<<64, 256, 0, n->stream>>>(kCin[l], kCout[l], cinT, n->params + n->wOff[l], n->wf[l],
                                                  l > 0 ? n->wt[l] : nullptr);
    }
    return net_fail(n, cudaGetLastError(), "cast weights");
}

}  // namespace

extern "C" {

int64_t ewg_net_num_params(void) {
    int64_t s = 0;
    for (int l = 0; l < kNetLayers; ++l) s += layer_w(l) + kCout[l];
    return s;
}

ewg_status ewg_net_create(uint64_t seed, ewg_net** out) {
    if (!out) return EWG_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { cudaGetLastError(); return EWG_ERR_NO_DEVICE; }
    ewg_net* n = new ewg_net();
    cudaGetDevice(&n->device);
    cudaError_t e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
    if (!e) e = conv_smem_attrs();
    int64_t off = 0;
    for (int l = 0; l < kNetLayers; ++l) {
        n->wOff[l] = off; off += layer_w(l);
        n->bOff[l] = off; off += kCout[l];
    }
    n->nParams = off;
    // He initialisation of the real (unpadded) weights; padded entries stay zero
    std::vector<float> h(off, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < kNetLayers; ++l) {
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (kTaps * kCinReal[l])) * (l == 3 ? 0.1f : 1.f));
        for (int tap = 0; tap < kTaps; ++tap)
            for (int co = 0; co < kCoutReal[l]; ++co)
                for (int ci = 0; ci < kCinReal[l]; ++ci)
                    h[n->wOff[l] + ((size_t)tap * kCout[l] + co) * kCin[l] + ci] = nd(rng);
    }
    if (!e) e = cudaMalloc(&n->params, sizeof(float) * off);
    if (!e) e = cudaMalloc(&n->grads, sizeof(float) * off);
    if (!e) e = cudaMalloc(&n->adamM, sizeof(float) * off);
    if (!e) e = cudaMalloc(&n->adamV, sizeof(float) * off);
    if (!e) e = cudaMalloc(&n->dLoss, sizeof(float));
    for (int l = 0; l < kNetLayers && !e; ++l) {
        e = cudaMalloc(&n->wf[l], sizeof(__nv_bfloat16) * layer_w(l));
        if (!e && l > 0) {
            const int cinT = kCout[l] == 8 ? 16 : kCout[l];
            e = cudaMalloc(&n->wt[l], sizeof(__nv_bfloat16) * kTaps * kCin[l] * cinT);
            if (!e) e = cudaMemsetAsync(n->wt[l], 0, sizeof(__nv_bfloat16) * kTaps * kCin[l] * cinT, n->stream);
        }
    }
    if (!e) e = cudaMemcpyAsync(n->params, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice, n->stream);
    if (!e) e = cudaMemsetAsync(n->adamM, 0, sizeof(float) * off, n->stream);
    if (!e) e = cudaMemsetAsync(n->adamV, 0, sizeof(float) * off, n->stream);
    if (!e) e = cudaStreamSynchronize(n->stream);
    if (e) {
        ewg_net_destroy(n);
        return EWG_ERR_CUDA;
    }
    refresh_weights(n);
    if (cudaStreamSynchronize(n->stream) != cudaSuccess) { ewg_net_destroy(n); return EWG_ERR_CUDA; }
    *out = n;
    return EWG_OK;
}

void ewg_net_destroy(ewg_net* n) {
    if (!n) return;
    if (n->stream) cudaStreamSynchronize(n->stream);
    void* ps[] = {n->params, n->grads, n->adamM, n->adamV, n->dLoss, n->act[0], n->act[1], n->act[2], n->act[3],
                  n->out, n->grad16, n->gradA, n->gradB, n->target};
    for (void* p : ps) if (p) cudaFree(p);
    for (int l = 0; l < kNetLayers; ++l) {
        if (n->wf[l]) cudaFree(n->wf[l]);
        if (n->wt[l]) cudaFree(n->wt[l]);
    }
    for (auto& s : n->samples) { cudaFree(s.f); cudaFree(s.t); }
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

const char* ewg_net_last_error(const ewg_net* n) { return n ? n->err.c_str() : "null net"; }

ewg_status ewg_net_get_params(ewg_net* n, float* host, int64_t count) {
    if (!n || !host || count != n->nParams) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(host, n->params, sizeof(float) * count, cudaMemcpyDeviceToHost, n->stream);
    if (!e) e = cudaStreamSynchronize(n->stream);
    return net_fail(n, e, "get params");
}

ewg_status ewg_net_set_params(ewg_net* n, const float* host, int64_t count) {
    if (!n || !host || count != n->nParams) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(n->params, host, sizeof(float) * count, cudaMemcpyHostToDevice, n->stream);
    if (e) return net_fail(n, e, "set params");
    ewg_status st = refresh_weights(n);
    if (st) return st;
    return net_fail(n, cudaStreamSynchronize(n->stream), "set params");
}

ewg_status ewg_net_set_scales(ewg_net* n, const double* s /* pScale, lnKMean, lnKScale, phiMean, phiScale, dtScale, tp, ts */) {
    if (!n || !s) return EWG_ERR_INVALID;
    n->fs = FeatureScales{s[0], s[1], s[2], s[3], s[4], s[5]};
    n->tp = s[6];
    n->ts = s[7];
    return EWG_OK;
}

ewg_status ewg_net_set_options(ewg_net* n, float lossWeightP, float lossWeightS, int32_t applyPressure,
                               double snThreshold) {
    if (!n || lossWeightP < 0 || lossWeightS < 0 || snThreshold < 0) return EWG_ERR_INVALID;
    n->wFront = lossWeightS > 1.f ? lossWeightS : 1.f;
    n->lossW[0] = lossWeightP;
    n->lossW[1] = lossWeightS;
    n->applyPressure = applyPressure != 0;
    n->snThreshold = snThreshold;
    return EWG_OK;
}

ewg_status ewg_net_get_scales(ewg_net* n, double* s) {
    if (!n || !s) return EWG_ERR_INVALID;
    const double v[8] = {n->fs.pScale, n->fs.lnKMean, n->fs.lnKScale, n->fs.phiMean, n->fs.phiScale, n->fs.dtScale, n->tp, n->ts};
    memcpy(s, v, sizeof(v));
    return EWG_OK;
}

// Forward and (optionally) backward on host data: features [B][D][H][W][5] (natural order per
// volume), targets [..][2]. Returns outputs [..][2], the MSE loss and, with grads != NULL, dL/dparams.
ewg_status ewg_net_eval_host(ewg_net* n, int32_t B, int32_t D, int32_t H, int32_t W, const float* feat,
                             const float* target, float* outY, float* loss, float* grads) {
    if (!n || !feat || B < 1 || D < 1 || H < 1 || W < 1) return EWG_ERR_INVALID;
    VolDims d{D, H, W, B};
    const int64_t V = d.V();
    ewg_status st = ensure_capacity(n, V);
    if (st) return st;
    std::vector<__nv_bfloat16> f16((size_t)V * 16);
    for (int64_t v = 0; v < V; ++v)
        for (int k = 0; k < 16; ++k) f16[v * 16 + k] = __float2bfloat16(k < 5 ? feat[v * 5 + k] : 0.f);
    cudaError_t e = cudaMemcpyAsync(n->act[0], f16.data(), sizeof(__nv_bfloat16) * V * 16, cudaMemcpyHostToDevice, n->stream);
    if (e) return net_fail(n, e, "upload features");
    if ((st = forward(n, d))) return st;
    if (target) {
        e = cudaMemcpyAsync(n->target, target, sizeof(float) * V * 2, cudaMemcpyHostToDevice, n->stream);
        if (!e) e = cudaMemsetAsync(n->dLoss, 0, sizeof(float), n->stream);
        if (e) return net_fail(n, e, "upload targets");
        k_mse<<<256, 256, 0, n->stream>>>(V, n->out, n->target, n->grad16, n->dLoss, n->lossW[0], n->lossW[1], n->act[0], n->wFront);
        if (grads) {
            if ((e = cudaMemsetAsync(n->grads, 0, sizeof(float) * n->nParams, n->stream))) return net_fail(n, e, "zero grads");
            if ((st = backward(n, d))) return st;
        }
    }
    if ((e = cudaGetLastError())) return net_fail(n, e, "net kernels");
    if (outY && (e = cudaMemcpyAsync(outY, n->out, sizeof(float) * V * 2, cudaMemcpyDeviceToHost, n->stream))) return net_fail(n, e, "read outputs");
    if (target && loss && (e = cudaMemcpyAsync(loss, n->dLoss, sizeof(float), cudaMemcpyDeviceToHost, n->stream))) return net_fail(n, e, "read loss");
    if (target && grads && (e = cudaMemcpyAsync(grads, n->grads, sizeof(float) * n->nParams, cudaMemcpyDeviceToHost, n->stream)))
        return net_fail(n, e, "read grads");
    if ((st = net_fail(n, cudaStreamSynchronize(n->stream), "sync net"))) return st;
    return conv_tc_check(&n->err);
}

// One 3x3x3 convolution layer on the tensor cores, synchronous on the stream (declared in ewg.h).
ewg_status ewg_net_conv3d(int32_t cin, int32_t epilogue, int32_t B, int32_t D, int32_t H, int32_t W, const void* in,
                          const void* w, const float* bias, const void* mask, void* out, void* stream) {
    if ((cin != 16 && cin != 32) || (epilogue != EPI_BIAS_RELU && epilogue != EPI_MASK) || B < 1 || D < 1 || H < 1 ||
        W < 1 || !in || !w || !out || (epilogue == EPI_BIAS_RELU && !bias) || (epilogue == EPI_MASK && !mask))
        return EWG_ERR_INVALID;
    for (const void* p : {in, w, (const void*)out, mask})
        if (p && (reinterpret_cast<uintptr_t>(p) & 15)) return EWG_ERR_INVALID;
    if (conv_tc_attrs() != cudaSuccess) { cudaGetLastError(); return EWG_ERR_CUDA; }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const VolDims d{D, H, W, B};
    const auto* x = static_cast<const __nv_bfloat16*>(in);
    const auto* wt = static_cast<const __nv_bfloat16*>(w);
    const auto* mk = static_cast<const __nv_bfloat16*>(mask);
    auto* y = static_cast<__nv_bfloat16*>(out);
    bool ok;
    if (cin == 16) {
        ok = epilogue == EPI_BIAS_RELU ? launch_conv_tc<16, 32, EPI_BIAS_RELU>(st, d, x, wt, bias, nullptr, 0, y, 32)
                                       : launch_conv_tc<16, 32, EPI_MASK>(st, d, x, wt, nullptr, mk, 32, y, 32);
    } else {
        ok = epilogue == EPI_BIAS_RELU ? launch_conv_tc<32, 32, EPI_BIAS_RELU>(st, d, x, wt, bias, nullptr, 0, y, 32)
                                       : launch_conv_tc<32, 32, EPI_MASK>(st, d, x, wt, nullptr, mk, 32, y, 32);
    }
    if (!ok) return EWG_ERR_CUDA;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return EWG_ERR_CUDA;
    return conv_tc_check(nullptr);
}

// Record one training sample from a context after a converged step: features of solution(1)
// (the state the step started from), target = solution(0) - solution(1). The context's grid is
// one volume.
ewg_status ewg_net_record_sample(ewg_net* n, ewg_ctx* ctx, double dt) {
    if (!n || !ctx) return EWG_ERR_INVALID;
    const Phys& P = ctx->P;
    ewg_net::Sample s{nullptr, nullptr, P.nz, P.ny, P.nx};
    cudaError_t e = cudaMalloc(&s.f, sizeof(__nv_bfloat16) * P.N * 16);
    if (!e) e = cudaMalloc(&s.t, sizeof(float) * P.N * 2);
    if (e) return net_fail(n, e, "alloc sample");
    cudaStreamSynchronize(n->stream);
    k_features<<<512, 256, 0, ctx->stream>>>(P, ctx->x1, ctx->perm, dt, n->fs, s.f);
    k_targets<<<512, 256, 0, ctx->stream>>>(P, ctx->x1, ctx->x0, n->tp, n->ts, s.t);
    e = cudaGetLastError();
    if (!e) e = cudaStreamSynchronize(ctx->stream);
    if (e) return net_fail(n, e, "record sample");
    n->samples.push_back(s);
    return EWG_OK;
}

int64_t ewg_net_num_samples(const ewg_net* n) { return n ? (int64_t)n->samples.size() : 0; }

// Adam steps on recorded samples (sample index list; each step one whole volume). Returns the
// mean loss of the steps.
ewg_status ewg_net_train(ewg_net* n, const int64_t* sampleIdx, int32_t steps, float lr, float* meanLoss) {
    if (!n || !sampleIdx || steps < 1) return EWG_ERR_INVALID;
    double acc = 0.0;
    for (int it = 0; it < steps; ++it) {
        const int64_t k = sampleIdx[it];
        if (k < 0 || k >= (int64_t)n->samples.size()) { n->err = "sample index out of range"; return EWG_ERR_INVALID; }
        const auto& s = n->samples[k];
        VolDims d{s.D, s.H, s.W, 1};
        const int64_t V = d.V();
        ewg_status st = ensure_capacity(n, V);
        if (st) return st;
        cudaError_t e = cudaMemcpyAsync(n->act[0], s.f, sizeof(__nv_bfloat16) * V * 16, cudaMemcpyDeviceToDevice, n->stream);
        if (!e) e = cudaMemsetAsync(n->dLoss, 0, sizeof(float), n->stream);
        if (!e) e = cudaMemsetAsync(n->grads, 0, sizeof(float) * n->nParams, n->stream);
        if (e) return net_fail(n, e, "train setup");
        if ((st = forward(n, d))) return st;
        k_mse<<<256, 256, 0, n->stream>>>(V, n->out, s.t, n->grad16, n->dLoss, n->lossW[0], n->lossW[1], n->act[0], n->wFront);
        if ((st = backward(n, d))) return st;
        n->adamStep += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)n->adamStep), c2 = 1.f - std::pow(b2, (float)n->adamStep);
        k_adam<<<128, 256, 0, n->stream>>>(n->nParams, n->params, n->grads, n->adamM, n->adamV, lr, b1, b2, 1e-8f, c1, c2);
        st = refresh_weights(n);
        if (st) return st;
        float l = 0.f;
        if ((e = cudaMemcpyAsync(&l, n->dLoss, sizeof(float), cudaMemcpyDeviceToHost, n->stream))) return net_fail(n, e, "loss");
        if ((e = cudaStreamSynchronize(n->stream))) return net_fail(n, e, "train sync");
        if ((st = conv_tc_check(&n->err))) return st;
        acc += l;
    }
    if (meanLoss) *meanLoss = (float)(acc / steps);
    return EWG_OK;
}

// Mean loss of recorded samples without updating the parameters.
ewg_status ewg_net_eval_samples(ewg_net* n, const int64_t* sampleIdx, int32_t count, float* meanLoss) {
    if (!n || !sampleIdx || count < 1) return EWG_ERR_INVALID;
    double acc = 0.0;
    for (int it = 0; it < count; ++it) {
        const auto& s = n->samples.at(sampleIdx[it]);
        VolDims d{s.D, s.H, s.W, 1};
        ewg_status st = ensure_capacity(n, d.V());
        if (st) return st;
        cudaMemcpyAsync(n->act[0], s.f, sizeof(__nv_bfloat16) * d.V() * 16, cudaMemcpyDeviceToDevice, n->stream);
        cudaMemsetAsync(n->dLoss, 0, sizeof(float), n->stream);
        if ((st = forward(n, d))) return st;
        k_mse<<<256, 256, 0, n->stream>>>(d.V(), n->out, s.t, n->grad16, n->dLoss, n->lossW[0], n->lossW[1], n->act[0], n->wFront);
        float l = 0.f;
        cudaMemcpyAsync(&l, n->dLoss, sizeof(float), cudaMemcpyDeviceToHost, n->stream);
        cudaError_t e = cudaStreamSynchronize(n->stream);
        if (e) return net_fail(n, e, "eval samples");
        if ((st = conv_tc_check(&n->err))) return st;
        acc += l;
    }
    if (meanLoss) *meanLoss = (float)(acc / count);
    return EWG_OK;
}

// Newton initial guess for the step of size dt starting from solution(1): run the network on the
// state, write the predicted solution(0), and keep it only if its residual max-norm is not larger
// than that of the previous-step guess (solution(1)); otherwise solution(0) = solution(1).
ewg_status ewg_predict_guess(ewg_ctx* ctx, ewg_net* n, double dt, int32_t* usedGuess, double* resGuess,
                             double* resPrev) {
    if (!ctx || !n) return EWG_ERR_INVALID;
    const Phys& P = ctx->P;
    VolDims d{P.nz, P.ny, P.nx, 1};
    ewg_status st = ensure_capacity(n, d.V());
    if (st) return st;
    cudaError_t e;
    // both the context and the network stream run this sequence; order them by synchronising
    if ((e = cudaStreamSynchronize(ctx->stream))) return cuda_fail(ctx, e, "sync ctx");
    k_features<<<512, 256, 0, n->stream>>>(P, ctx->x1, ctx->perm, dt, n->fs, n->act[0]);
    if ((st = forward(n, d))) return st;
    k_apply_guess<<<512, 256, 0, n->stream>>>(P, ctx->x1, n->out, n->tp, n->ts, n->applyPressure, n->snThreshold, ctx->x0);
    if ((e = cudaGetLastError())) return cuda_fail(ctx, e, "guess kernels");
    if ((e = cudaStreamSynchronize(n->stream))) return cuda_fail(ctx, e, "sync guess");
    if ((st = conv_tc_check(&n->err))) return st;
    double rg = 0.0, rp = 0.0;
    int bad = 0;
    // residual-only evaluations (the old-time storage is that of solution(1) in both)
    if ((st = launch_linearize(ctx, dt, false, ctx->x0, ctx->r, &rg, &bad))) return st;
    if (bad) rg = INFINITY;
    if ((st = launch_linearize(ctx, dt, false, ctx->x1, ctx->r, &rp, &bad))) return st;
    if (bad) rp = INFINITY;
    const bool use = rg <= rp;
    if (!use) {
        e = cudaMemcpyAsync(ctx->x0, ctx->x1, sizeof(double2) * P.N, cudaMemcpyDeviceToDevice, ctx->stream);
        if (!e) e = cudaStreamSynchronize(ctx->stream);
        if (e) return cuda_fail(ctx, e, "fallback copy");
    }
    if (usedGuess) *usedGuess = use ? 1 : 0;
    if (resGuess) *resGuess = rg;
    if (resPrev) *resPrev = rp;
    return EWG_OK;
}

}  // extern "C"

// ---- forward pass that allocates nothing ----------------------------------------------------
//
// ewg_net_forward_noalloc runs the same four convolution launches as the forward pass of
// ewg_net_eval_host (three on the tensor cores, whose tensor maps are host-side descriptors, and
// the 2-output layer), for callers that must not allocate device memory: a host simulator that
// hands all of the device's memory to its own arena up front, and time-step loops that cannot
// afford the device-wide synchronisation of cudaMalloc / cudaFree. The caller
// passes the FP32 parameters, the features and the output on the device; the BF16 weights, the
// 16-channel BF16 features and two 32-channel activation buffers live in one file-scope device
// array of fixed size, which every GPU that loads this library holds until the process exits.
namespace ewg {
namespace {

constexpr int64_t kNoAllocMaxVoxels = EWG_NET_NOALLOC_MAX_VOXELS;
constexpr int64_t kNoAllocWeights = (int64_t)kTaps * (16 * 32 + 32 * 32 + 32 * 32 + 32 * 8);
constexpr size_t kNoAllocOffFeat = (sizeof(__nv_bfloat16) * kNoAllocWeights + 255) / 256 * 256;
constexpr size_t kNoAllocOffActA = kNoAllocOffFeat + sizeof(__nv_bfloat16) * kNoAllocMaxVoxels * 16;
constexpr size_t kNoAllocOffActB = kNoAllocOffActA + sizeof(__nv_bfloat16) * kNoAllocMaxVoxels * 32;
constexpr size_t kNoAllocBytes = kNoAllocOffActB + sizeof(__nv_bfloat16) * kNoAllocMaxVoxels * 32;
constexpr int kNoAllocMaxDevices = 64;

// The scratch. Its name in host code is only a handle for cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_netScratch[kNoAllocBytes];

std::mutex g_netScratchMutex;
unsigned char* g_netScratchPtr[kNoAllocMaxDevices] = {};

// features [V][5] FP32 -> [V][16] BF16, channels 5..15 zero (every word of the buffer the
// convolution reads for these V voxels is written here)
__global__ void k_pack_features(int64_t V, const float* __restrict__ f5, __nv_bfloat16* __restrict__ f16) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V * 16; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i >> 4;
        const int k = (int)(i & 15);
        f16[i] = __float2bfloat16(k < 5 ? f5[v * 5 + k] : 0.f);
    }
}

template <int CIN, int COUT, int EPI>
cudaError_t noalloc_conv_attr() {
    return cudaFuncSetAttribute(k_conv3d<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(__nv_bfloat16) * kTaps * COUT * CIN));
}

template <int CIN, int COUT, int EPI>
void noalloc_conv(cudaStream_t st, const VolDims& d, const __nv_bfloat16* in, const __nv_bfloat16* W,
                  const float* bias, void* out, int outC) {
    const size_t smem = sizeof(__nv_bfloat16) * kTaps * COUT * CIN;
    const int64_t tiles = (d.V() + 15) / 16;
    int64_t blocks = (tiles + 3) / 4;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_conv3d<CIN, COUT, EPI><<<(int)blocks, 128, smem, st>>>(d, in, W, bias, nullptr, 0, out, outC);
}

ewg_status noalloc_fail(char* msg, int32_t len, ewg_status st, const char* text) {
    if (msg && len > 0) std::snprintf(msg, (size_t)len, "%s", text);
    return st;
}

// Once per device, with that device current: the scratch's device address and the kernels'
// shared-memory limits.
ewg_status noalloc_setup(int dev, unsigned char** out, char* msg, int32_t len) {
    std::lock_guard<std::mutex> lock(g_netScratchMutex);
    if (!g_netScratchPtr[dev]) {
        unsigned char* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_netScratch);
        if (e == cudaSuccess) e = noalloc_conv_attr<16, 32, EPI_BIAS_RELU>();
        if (e == cudaSuccess) e = noalloc_conv_attr<32, 32, EPI_BIAS_RELU>();
        if (e == cudaSuccess) e = noalloc_conv_attr<32, 8, EPI_BIAS>();
        if (e == cudaSuccess) e = conv_tc_attrs();
        if (e != cudaSuccess) {
            char text[256];
            std::snprintf(text, sizeof(text), "no-allocation scratch set-up: %s", cudaGetErrorString(e));
            return noalloc_fail(msg, len, EWG_ERR_CUDA, text);
        }
        g_netScratchPtr[dev] = ptr;
    }
    *out = g_netScratchPtr[dev];
    return EWG_OK;
}

}  // namespace
}  // namespace ewg

extern "C" ewg_status ewg_net_forward_noalloc(const float* params, int32_t B, int32_t D, int32_t H, int32_t W,
                                              const float* features, float* outputs, void* stream, char* message,
                                              int32_t message_len) {
    if (message && message_len > 0) message[0] = '\0';
    if (!params || !features || !outputs || B < 1 || D < 1 || H < 1 || W < 1)
        return noalloc_fail(message, message_len, EWG_ERR_INVALID, "null pointer or non-positive extent");
    VolDims d{D, H, W, B};
    const int64_t V = d.V();
    if (V > kNoAllocMaxVoxels) {
        char text[256];
        std::snprintf(text, sizeof(text),
                      "batch of %lld voxels exceeds the no-allocation limit of %lld voxels (B*D*H*W)",
                      (long long)V, (long long)kNoAllocMaxVoxels);
        return noalloc_fail(message, message_len, EWG_ERR_INVALID, text);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(message, message_len, EWG_ERR_NO_DEVICE, cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return noalloc_fail(message, message_len, EWG_ERR_INVALID, "device ordinal above 63");
    unsigned char* base = nullptr;
    ewg_status st = noalloc_setup(dev, &base, message, message_len);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    __nv_bfloat16* wf[kNetLayers];
    int64_t woff = 0, poff = 0, boff[kNetLayers];
    for (int l = 0; l < kNetLayers; ++l) {
        wf[l] = reinterpret_cast<__nv_bfloat16*>(base) + woff;
        k_cast_weights<<<64, 256, 0, s>>>(kCin[l], kCout[l], kCout[l], params + poff, wf[l], nullptr);
        woff += layer_w(l);
        boff[l] = poff + layer_w(l);
        poff = boff[l] + kCout[l];
    }
    __nv_bfloat16* feat = reinterpret_cast<__nv_bfloat16*>(base + kNoAllocOffFeat);
    __nv_bfloat16* actA = reinterpret_cast<__nv_bfloat16*>(base + kNoAllocOffActA);
    __nv_bfloat16* actB = reinterpret_cast<__nv_bfloat16*>(base + kNoAllocOffActB);
    k_pack_features<<<256, 256, 0, s>>>(V, features, feat);
    bool ok = launch_conv_tc<16, 32, EPI_BIAS_RELU>(s, d, feat, wf[0], params + boff[0], nullptr, 0, actA, 32);
    ok = ok && launch_conv_tc<32, 32, EPI_BIAS_RELU>(s, d, actA, wf[1], params + boff[1], nullptr, 0, actB, 32);
    ok = ok && launch_conv_tc<32, 32, EPI_BIAS_RELU>(s, d, actB, wf[2], params + boff[2], nullptr, 0, actA, 32);
    if (!ok) return noalloc_fail(message, message_len, EWG_ERR_CUDA, "tensor map of a convolution could not be built");
    noalloc_conv<32, 8, EPI_BIAS>(s, d, actA, wf[3], params + boff[3], outputs, 2);
    if ((e = cudaGetLastError()) != cudaSuccess) return noalloc_fail(message, message_len, EWG_ERR_CUDA, cudaGetErrorString(e));
    return EWG_OK;
}
