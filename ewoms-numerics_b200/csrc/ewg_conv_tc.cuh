// 3x3x3 convolution of the guess network on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Implicit GEMM per tile of 128 output voxels (a 32 x 4 patch of one z-plane of one volume):
//   D[128 voxels][COUT] = sum over the 27 taps of A_tap[128][CIN] * W_tap[CIN][COUT]
// with A_tap the input patch shifted by the tap, loaded by TMA from a 5-D tensor map over the
// channels-last activations (C, x, y, z, volume): the shifted box may reach outside the volume,
// where TMA fills zeros, which is the convolution's zero padding. Operands are K-major BF16 in
// shared memory with the TMA / UMMA swizzle of their row length (64 B rows for 32 channels, 32 B
// rows for 16), the accumulator is FP32 in tensor memory (128 lanes = voxels, COUT columns).
//
// One CTA of 192 threads is persistent over tiles:
//   warp 4 (one lane)  TMA producer: the 27 weight taps once, then per tile and tap one A box
//                      into a ring of kTcStages stages (mbarriers full / empty);
//   warp 5 (one lane)  MMA issuer: per tap CIN / 16 tcgen05.mma (M = 128, N = COUT, K = 16) into
//                      one of two TMEM accumulators, tcgen05.commit releasing the stage, and after
//                      the last tap one committing the accumulator (mbarriers accFull / accEmpty);
//   warps 0-3          epilogue: tcgen05.ld of the accumulator lanes 32w .. 32w + 31 (warp w, one
//                      voxel per thread), release of the accumulator, bias + ReLU or the ReLU mask
//                      of the layer below, BF16 store of the voxel's COUT channels.
// The two accumulators let the MMAs of tile i + 1 run while the epilogue drains tile i.
// Every mbarrier wait is bounded: past kTcSpinLimit polls the kernel records the stage that gave
// up in *err and every role leaves its loop; the CTA then waits (bounded) for its own MMAs and
// copies in flight and frees its tensor memory before it exits.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace ewg {

constexpr int kTcThreads = 192;
constexpr int kTcStages = 6;
constexpr int kTcTileX = 32, kTcTileY = 4, kTcRows = 128;
constexpr int kTcTmemCols = 64;          // two accumulators of up to 32 FP32 columns
constexpr uint32_t kTcSpinLimit = 1u << 22;

// error codes written to *err (the first one wins)
constexpr int TC_ERR_FULL = 1, TC_ERR_EMPTY = 2, TC_ERR_ACC_FULL = 3, TC_ERR_ACC_EMPTY = 4, TC_ERR_WEIGHTS = 5,
              TC_ERR_DRAIN = 6;

template <int CIN, int COUT>
struct TcShape {
    static constexpr int rowBytes = CIN * 2;                   // one voxel's (or weight row's) channels
    static constexpr int aBytes = kTcRows * rowBytes;          // one A stage
    static constexpr int wTapBytes = COUT * rowBytes;          // one tap's weights
    static constexpr int wBytes = 27 * wTapBytes;
    static constexpr int kSteps = CIN / 16;                    // MMAs per tap
    // shared memory: weights, A stages (each 1024-byte aligned), barriers, TMEM slot
    static constexpr int wRegion = (wBytes + 1023) / 1024 * 1024;
    static constexpr int aRegion = (aBytes + 1023) / 1024 * 1024;
    static constexpr int barOff = wRegion + kTcStages * aRegion;
    static constexpr int smemBytes = barOff + 256 + 1024;      // + barriers, + alignment slack
    // UMMA / TMA swizzle of the row length: 64 B -> SWIZZLE_64B (descriptor layout 4), 32 B ->
    // SWIZZLE_32B (layout 6); the swizzle atom is 8 rows, so the stride between 8-row groups
    // (SBO) is 8 rows.
    static constexpr uint64_t layoutType = rowBytes == 64 ? 4ull : 6ull;
    static constexpr uint64_t sbo16 = 8 * rowBytes / 16;
    static_assert(CIN == 16 || CIN == 32, "CIN 16 or 32");
    static_assert(COUT % 16 == 0 && COUT >= 16 && COUT <= 32, "COUT 16 or 32");
};

// Shared-memory matrix descriptor of a K-major swizzled operand (PTX ISA, tcgen05 matrix
// descriptor): start address >> 4 in bits 0-13, leading byte offset >> 4 in 16-29 (1 for
// swizzled K-major layouts), stride byte offset >> 4 in 32-45, version 1 in 46-47, base offset 0
// (stages are 1024-byte aligned), layout type in 61-63.
template <int CIN, int COUT>
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr) {
    using S = TcShape<CIN, COUT>;
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | (1ull << 16) | (S::sbo16 << 32) | (1ull << 46) |
           (S::layoutType << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (7-9 = 1,
// 10-12 = 1), both K-major, N >> 3 in 17-22, M >> 4 in 24-28.
template <int N>
__host__ __device__ constexpr uint32_t tc_instr_desc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void tc_bar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tc_bar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc_smem_u32(bar)) : "memory");
}

// waits until the phase of the given parity has completed; false after kTcSpinLimit polls
__device__ __forceinline__ bool tc_bar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = tc_smem_u32(bar);
    for (uint32_t i = 0; i < kTcSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fail(int* err, int* dead, int code) {
    atomicCAS(err, 0, code);
    *(volatile int*)dead = 1;
}
__device__ __forceinline__ bool tc_dead(const int* dead) { return *(const volatile int*)dead != 0; }

// TMA: one tile box of a tensor map into shared memory, completing on bar
__device__ __forceinline__ void tc_tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                               int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6, %7}], [%2];"
        ::"r"(tc_smem_u32(dst)), "l"(map), "r"(tc_smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}
__device__ __forceinline__ void tc_tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(tc_smem_u32(dst)), "l"(map), "r"(tc_smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}
__device__ __forceinline__ void tc_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// tensor memory: allocation by one whole warp (address written to *slot), release, free
__device__ __forceinline__ void tc_tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// D (tmem) (+)= A (smem desc) * B (smem desc); accumulate = false overwrites D
__device__ __forceinline__ void tc_mma_f16(uint32_t tmemD, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                           bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmemD), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
// bar completes one arrival when every MMA issued so far by this thread has completed
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (lane = thread)
__device__ __forceinline__ void tc_tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
// 16 consecutive FP32 columns
__device__ __forceinline__ void tc_tmem_ld16(uint32_t taddr, float (&v)[32]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
#pragma unroll
    for (int i = 16; i < 32; ++i) v[i] = 0.f;
}

__device__ __forceinline__ void tc_fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

struct TcTile {
    int b, z, y0, x0;
};
// tile t of the volume batch: x fastest, then y, z, volume
__device__ __forceinline__ TcTile tc_tile(const int D, const int H, const int W, int64_t t) {
    const int nx = (W + kTcTileX - 1) / kTcTileX, ny = (H + kTcTileY - 1) / kTcTileY;
    TcTile r;
    r.x0 = (int)(t % nx) * kTcTileX;
    t /= nx;
    r.y0 = (int)(t % ny) * kTcTileY;
    t /= ny;
    r.z = (int)(t % D);
    r.b = (int)(t / D);
    return r;
}

// EPI 0: y = relu(acc + bias); EPI 2: y = acc * (mask > 0) (mask: the layer below, maskC channels)
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1) k_conv3d_tc(const __grid_constant__ CUtensorMap mapIn,
                                                             const __grid_constant__ CUtensorMap mapW, int D, int H,
                                                             int W, int64_t nTiles, const float* __restrict__ bias,
                                                             const __nv_bfloat16* __restrict__ mask, int maskC,
                                                             __nv_bfloat16* __restrict__ out, int outC,
                                                             int* __restrict__ err) {
    using S = TcShape<CIN, COUT>;
    extern __shared__ unsigned char smemRaw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smemRaw + 1023) & ~(uintptr_t)1023);
    unsigned char* wS = smem;
    unsigned char* aS = smem + S::wRegion;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::barOff);
    uint64_t* full = bars;                     // [kTcStages]
    uint64_t* empty = bars + kTcStages;        // [kTcStages]
    uint64_t* accFull = bars + 2 * kTcStages;  // [2]
    uint64_t* accEmpty = accFull + 2;          // [2]
    uint64_t* wBar = accEmpty + 2;
    uint64_t* drain = wBar + 1;
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(drain + 1);
    int* dead = reinterpret_cast<int*>(tmemSlot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kTcStages; ++i) {
            tc_bar_init(&full[i], 1);
            tc_bar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc_bar_init(&accFull[i], 1);
            tc_bar_init(&accEmpty[i], 128);
        }
        tc_bar_init(wBar, 1);
        tc_bar_init(drain, 1);
        *dead = 0;
        tc_fence_barrier_init();
    }
    if (warp == 0) tc_tmem_alloc(tmemSlot, kTcTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;

    if (warp == 4 && lane == 0) {
        // ---- TMA producer
        tc_prefetch_map(&mapIn);
        tc_prefetch_map(&mapW);
        tc_bar_expect_tx(wBar, S::wBytes);
        for (int tap = 0; tap < 27; ++tap) tc_tma_load_2d(wS + tap * S::wTapBytes, &mapW, wBar, 0, tap * COUT);
        uint32_t it = 0;
        for (int64_t t = blockIdx.x; t < nTiles && !tc_dead(dead); t += gridDim.x) {
            const TcTile tl = tc_tile(D, H, W, t);
            for (int tap = 0; tap < 27; ++tap, ++it) {
                const uint32_t st = it % kTcStages, ph = (it / kTcStages) & 1;
                if (it >= (uint32_t)kTcStages && !tc_bar_wait(&empty[st], ph ^ 1)) {
                    tc_fail(err, dead, TC_ERR_EMPTY);
                    break;
                }
                const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
                tc_bar_expect_tx(&full[st], S::aBytes);
                tc_tma_load_5d(aS + st * S::aRegion, &mapIn, &full[st], 0, tl.x0 + dx, tl.y0 + dy, tl.z + dz, tl.b);
            }
        }
        // the copies still in flight (normally none: the MMA warp consumed every stage)
        const uint32_t issued = it;
        for (uint32_t k = issued > (uint32_t)kTcStages ? issued - kTcStages : 0; k < issued; ++k)
            if (!tc_bar_wait(&full[k % kTcStages], (k / kTcStages) & 1)) { tc_fail(err, dead, TC_ERR_DRAIN); break; }
        if (!tc_bar_wait(wBar, 0)) tc_fail(err, dead, TC_ERR_DRAIN);
    } else if (warp == 5 && lane == 0) {
        // ---- MMA issuer
        constexpr uint32_t idesc = tc_instr_desc<COUT>();
        const uint32_t wBase = tc_smem_u32(wS), aBase = tc_smem_u32(aS);
        bool ok = tc_bar_wait(wBar, 0);
        if (!ok) tc_fail(err, dead, TC_ERR_WEIGHTS);
        tc_fence_after();
        uint32_t it = 0, local = 0;
        for (int64_t t = blockIdx.x; ok && t < nTiles && !tc_dead(dead); t += gridDim.x, ++local) {
            const uint32_t acc = local & 1, accPh = (local >> 1) & 1;
            if (local >= 2 && !tc_bar_wait(&accEmpty[acc], accPh ^ 1)) {
                tc_fail(err, dead, TC_ERR_ACC_EMPTY);
                break;
            }
            tc_fence_after();
            const uint32_t d = tmem + acc * 32;
            for (int tap = 0; tap < 27; ++tap, ++it) {
                const uint32_t st = it % kTcStages, ph = (it / kTcStages) & 1;
                if (!tc_bar_wait(&full[st], ph)) {
                    tc_fail(err, dead, TC_ERR_FULL);
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int k = 0; k < S::kSteps; ++k) {
                    const uint64_t ad = tc_smem_desc<CIN, COUT>(aBase + st * S::aRegion + k * 32);
                    const uint64_t bd = tc_smem_desc<CIN, COUT>(wBase + tap * S::wTapBytes + k * 32);
                    tc_mma_f16(d, ad, bd, idesc, tap > 0 || k > 0);
                }
                tc_commit(&empty[st]);
            }
            if (!ok) break;
            tc_commit(&accFull[acc]);
        }
        // every MMA issued has completed before the tensor memory is freed
        tc_commit(drain);
        if (!tc_bar_wait(drain, 0)) tc_fail(err, dead, TC_ERR_DRAIN);
    } else if (warp < 4) {
        // ---- epilogue: thread = voxel row 32 warp + lane of the tile
        float bv[COUT];
#pragma unroll
        for (int c = 0; c < COUT; ++c) bv[c] = EPI == 0 ? bias[c] : 0.f;
        const int row = warp * 32 + lane, rx = row % kTcTileX, ry = row / kTcTileX;
        uint32_t local = 0;
        for (int64_t t = blockIdx.x; t < nTiles; t += gridDim.x, ++local) {
            const uint32_t acc = local & 1, accPh = (local >> 1) & 1;
            // lane 0 waits and the warp follows it, so the warp stays converged for tcgen05.ld
            int stop = 0;
            if (lane == 0) stop = tc_dead(dead) ? 1 : (tc_bar_wait(&accFull[acc], accPh) ? 0 : 2);
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop == 2 && lane == 0) tc_fail(err, dead, TC_ERR_ACC_FULL);
            if (stop) break;
            tc_fence_after();
            float v[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + acc * 32;
            if (COUT == 32) tc_tmem_ld32(taddr, v);
            else tc_tmem_ld16(taddr, v);
            tc_fence_before();
            tc_bar_arrive(&accEmpty[acc]);
            const TcTile tl = tc_tile(D, H, W, t);
            const int x = tl.x0 + rx, y = tl.y0 + ry;
            if (x >= W || y >= H) continue;
            const int64_t vox = (((int64_t)tl.b * D + tl.z) * H + y) * W + x;
            if (EPI == 2) {
                const uint4* mp = reinterpret_cast<const uint4*>(mask + vox * maskC);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    const uint4 m4 = mp[q];
                    const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(&m4);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        if (!(__bfloat162float(mb[j]) > 0.f)) v[q * 8 + j] = 0.f;
                }
            } else {
#pragma unroll
                for (int c = 0; c < COUT; ++c) v[c] = fmaxf(v[c] + bv[c], 0.f);
            }
            uint4* op = reinterpret_cast<uint4*>(out + vox * outC);
#pragma unroll
            for (int q = 0; q < COUT / 8; ++q) {
                uint4 o;
                __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
                for (int j = 0; j < 4; ++j) ob[j] = __floats2bfloat162_rn(v[q * 8 + 2 * j], v[q * 8 + 2 * j + 1]);
                op[q] = o;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tc_tmem_free(tmem, kTcTmemCols);
    }
}

// ---- row tiles ------------------------------------------------------------------------------
//
// For volumes at least kTcRowMinW wide a tile is 128 consecutive voxels of one x-row; its input
// boxes are 130 x-positions (x0 - 1 .. x0 + 128) of one row, unswizzled: every position is one
// 16-byte row of 8 channels, so the A operand of tap dx is the same box read from position dx + 1
// (a K-major operand without swizzle whose 8-row core matrices are 128 B apart).
constexpr int kTcRowMinW = 96;
constexpr int kTcRowX = 130;

// ---- row tiles with a ring of input rows -----------------------------------------------------------
//
// A CTA walks segments of kTcSegRows consecutive output rows of one (x-tile, z, volume) column.
// Output row y needs the input rows y - 1, y, y + 1 of the planes z - 1, z, z + 1; consecutive
// output rows share two of the three, so the producer loads each input row once per segment: an
// "item" is one input row y' of the three planes (3 x CIN / 8 boxes of 8 channels x 130
// x-positions x 1 row, unswizzled) into one slot of a ring of kTcRingSlots. The MMA issuer runs
// output row y from the items of y - 1, y, y + 1 (the A operand of tap (dx, dy, dz) is the slot of
// row y + dy, plane z + dz, at x-offset dx + 1) and frees the item of row y - 1 after the row (a
// segment's last row frees all three). Per 128 output voxels the shared-memory fill is one item
// (3 x CIN / 8 x 2080 B, 25 KB for 32 channels) plus the segment's two extra rows.
constexpr int kTcSegRows = 16;
constexpr int kTcRingSlots = 4;
constexpr int kTcLineBytes = kTcRowX * 16;                         // one box: 130 positions x 16 B
constexpr int kTcLineStride = (kTcLineBytes + 127) / 128 * 128;    // 2176: boxes 128-byte aligned

template <int CIN, int COUT>
struct TcRingShape {
    using S = TcShape<CIN, COUT>;
    static constexpr int groups = CIN / 8;
    static constexpr int planeBytes = groups * kTcLineStride;      // one input row of one plane
    static constexpr int slotBytes = 3 * planeBytes;               // one item: the row in 3 planes
    static constexpr int txBytes = 3 * groups * kTcLineBytes;      // bytes an item's boxes deliver
    static constexpr int barOff = S::wRegion + kTcRingSlots * slotBytes;
    static constexpr int smemBytes = barOff + 256 + 1024;
};

// descriptor of an A operand in a ring slot: no swizzle, LBO = one 8-channel box, SBO = 8 rows
__device__ __forceinline__ uint64_t tc_smem_desc_line(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(kTcLineStride >> 4) << 16) |
           ((uint64_t)(128 >> 4) << 32) | (1ull << 46);
}

struct TcSeg {
    int b, z, y0, y1, x0;  // output rows y0 .. y1 - 1 of the column (b, z, x0 .. x0 + 127)
};
__device__ __forceinline__ TcSeg tc_seg(const int D, const int H, const int W, int64_t sIdx) {
    const int nx = (W + kTcRows - 1) / kTcRows, ns = (H + kTcSegRows - 1) / kTcSegRows;
    TcSeg r;
    r.x0 = (int)(sIdx % nx) * kTcRows;
    sIdx /= nx;
    r.y0 = (int)(sIdx % ns) * kTcSegRows;
    sIdx /= ns;
    r.z = (int)(sIdx % D);
    r.b = (int)(sIdx / D);
    r.y1 = r.y0 + kTcSegRows < H ? r.y0 + kTcSegRows : H;
    return r;
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1) k_conv3d_tc_ring(const __grid_constant__ CUtensorMap mapIn,
                                                                  const __grid_constant__ CUtensorMap mapW, int D, int H,
                                                                  int W, int64_t nSegs, const float* __restrict__ bias,
                                                                  const __nv_bfloat16* __restrict__ mask, int maskC,
                                                                  __nv_bfloat16* __restrict__ out, int outC,
                                                                  int* __restrict__ err) {
    using S = TcShape<CIN, COUT>;
    using R = TcRingShape<CIN, COUT>;
    constexpr int NS = kTcRingSlots;
    extern __shared__ unsigned char smemRaw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smemRaw + 1023) & ~(uintptr_t)1023);
    unsigned char* wS = smem;
    unsigned char* aS = smem + S::wRegion;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + R::barOff);
    uint64_t* full = bars;               // [NS]
    uint64_t* empty = bars + NS;         // [NS]
    uint64_t* accFull = bars + 2 * NS;   // [2]
    uint64_t* accEmpty = accFull + 2;    // [2]
    uint64_t* wBar = accEmpty + 2;
    uint64_t* drain = wBar + 1;
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(drain + 1);
    int* dead = reinterpret_cast<int*>(tmemSlot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) {
            tc_bar_init(&full[i], 1);
            tc_bar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            tc_bar_init(&accFull[i], 1);
            tc_bar_init(&accEmpty[i], 128);
        }
        tc_bar_init(wBar, 1);
        tc_bar_init(drain, 1);
        *dead = 0;
        tc_fence_barrier_init();
    }
    if (warp == 0) tc_tmem_alloc(tmemSlot, kTcTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmemSlot;

    if (warp == 4 && lane == 0) {
        // ---- TMA producer: weights, then per segment the input rows y0 - 1 .. y1 as items
        tc_prefetch_map(&mapIn);
        tc_prefetch_map(&mapW);
        tc_bar_expect_tx(wBar, S::wBytes);
        for (int tap = 0; tap < 27; ++tap) tc_tma_load_2d(wS + tap * S::wTapBytes, &mapW, wBar, 0, tap * COUT);
        uint32_t it = 0;
        bool stop = false;
        for (int64_t sg = blockIdx.x; sg < nSegs && !stop && !tc_dead(dead); sg += gridDim.x) {
            const TcSeg seg = tc_seg(D, H, W, sg);
            for (int yi = seg.y0 - 1; yi <= seg.y1; ++yi, ++it) {
                const uint32_t st = it % NS, ph = (it / NS) & 1;
                if (it >= (uint32_t)NS && !tc_bar_wait(&empty[st], ph ^ 1)) {
                    tc_fail(err, dead, TC_ERR_EMPTY);
                    stop = true;
                    break;
                }
                tc_bar_expect_tx(&full[st], R::txBytes);
                unsigned char* slot = aS + st * R::slotBytes;
#pragma unroll
                for (int pz = 0; pz < 3; ++pz)
#pragma unroll
                    for (int g = 0; g < R::groups; ++g)
                        tc_tma_load_5d(slot + pz * R::planeBytes + g * kTcLineStride, &mapIn, &full[st], 8 * g,
                                       seg.x0 - 1, yi, seg.z + pz - 1, seg.b);
            }
        }
        const uint32_t issued = it;
        for (uint32_t k = issued > (uint32_t)NS ? issued - NS : 0; k < issued; ++k)
            if (!tc_bar_wait(&full[k % NS], (k / NS) & 1)) { tc_fail(err, dead, TC_ERR_DRAIN); break; }
        if (!tc_bar_wait(wBar, 0)) tc_fail(err, dead, TC_ERR_DRAIN);
    } else if (warp == 5 && lane == 0) {
        // ---- MMA issuer: output row y from the items of rows y - 1, y, y + 1
        constexpr uint32_t idesc = tc_instr_desc<COUT>();
        const uint32_t wBase = tc_smem_u32(wS), aBase = tc_smem_u32(aS);
        bool ok = tc_bar_wait(wBar, 0);
        if (!ok) tc_fail(err, dead, TC_ERR_WEIGHTS);
        tc_fence_after();
        uint32_t item0 = 0, local = 0;  // first item of the segment, output rows done
        for (int64_t sg = blockIdx.x; ok && sg < nSegs && !tc_dead(dead); sg += gridDim.x) {
            const TcSeg seg = tc_seg(D, H, W, sg);
            const int rows = seg.y1 - seg.y0;
            // the segment's first two items
            for (uint32_t k = item0; k < item0 + 2 && ok; ++k) {
                if (!tc_bar_wait(&full[k % NS], (k / NS) & 1)) { tc_fail(err, dead, TC_ERR_FULL); ok = false; }
            }
            for (int j = 0; j < rows && ok; ++j, ++local) {
                const uint32_t acc = local & 1, accPh = (local >> 1) & 1;
                if (local >= 2 && !tc_bar_wait(&accEmpty[acc], accPh ^ 1)) {
                    tc_fail(err, dead, TC_ERR_ACC_EMPTY);
                    ok = false;
                    break;
                }
                const uint32_t knew = item0 + j + 2;  // input row y + 1
                if (!tc_bar_wait(&full[knew % NS], (knew / NS) & 1)) {
                    tc_fail(err, dead, TC_ERR_FULL);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + acc * 32;
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
                    const uint32_t slot = aBase + ((item0 + j + dy) % NS) * R::slotBytes;
#pragma unroll
                    for (int pz = 0; pz < 3; ++pz)
#pragma unroll
                        for (int dx = 0; dx < 3; ++dx) {
                            const int tap = pz * 9 + dy * 3 + dx;  // 9 (dz + 1) + 3 (dy + 1) + dx + 1
#pragma unroll
                            for (int k = 0; k < S::kSteps; ++k) {
                                const uint64_t ad =
                                    tc_smem_desc_line(slot + pz * R::planeBytes + 2 * k * kTcLineStride + dx * 16);
                                const uint64_t bd = tc_smem_desc<CIN, COUT>(wBase + tap * S::wTapBytes + k * 32);
                                tc_mma_f16(d, ad, bd, idesc, tap > 0 || k > 0);
                            }
                        }
                }
                tc_commit(&accFull[acc]);
                // input row y - 1 is done; after the segment's last row, rows y and y + 1 too
                tc_commit(&empty[(item0 + j) % NS]);
                if (j == rows - 1) {
                    tc_commit(&empty[(item0 + j + 1) % NS]);
                    tc_commit(&empty[(item0 + j + 2) % NS]);
                }
            }
            item0 += rows + 2;
        }
        tc_commit(drain);
        if (!tc_bar_wait(drain, 0)) tc_fail(err, dead, TC_ERR_DRAIN);
    } else if (warp < 4) {
        // ---- epilogue: thread = voxel x0 + 32 warp + lane of the output row
        float bv[COUT];
#pragma unroll
        for (int c = 0; c < COUT; ++c) bv[c] = EPI == 0 ? bias[c] : 0.f;
        const int row = warp * 32 + lane;
        uint32_t local = 0;
        bool go = true;
        for (int64_t sg = blockIdx.x; go && sg < nSegs; sg += gridDim.x) {
            const TcSeg seg = tc_seg(D, H, W, sg);
            for (int y = seg.y0; y < seg.y1; ++y, ++local) {
                const uint32_t acc = local & 1, accPh = (local >> 1) & 1;
                int stop = 0;
                if (lane == 0) stop = tc_dead(dead) ? 1 : (tc_bar_wait(&accFull[acc], accPh) ? 0 : 2);
                stop = __shfl_sync(0xffffffffu, stop, 0);
                if (stop == 2 && lane == 0) tc_fail(err, dead, TC_ERR_ACC_FULL);
                if (stop) {
                    go = false;
                    break;
                }
                tc_fence_after();
                float v[32];
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + acc * 32;
                if (COUT == 32) tc_tmem_ld32(taddr, v);
                else tc_tmem_ld16(taddr, v);
                tc_fence_before();
                tc_bar_arrive(&accEmpty[acc]);
                const int x = seg.x0 + row;
                if (x >= W) continue;
                const int64_t vox = (((int64_t)seg.b * D + seg.z) * H + y) * W + x;
                if (EPI == 2) {
                    const uint4* mp = reinterpret_cast<const uint4*>(mask + vox * maskC);
#pragma unroll
                    for (int q = 0; q < COUT / 8; ++q) {
                        const uint4 m4 = mp[q];
                        const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(&m4);
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj)
                            if (!(__bfloat162float(mb[jj]) > 0.f)) v[q * 8 + jj] = 0.f;
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < COUT; ++c) v[c] = fmaxf(v[c] + bv[c], 0.f);
                }
                uint4* op = reinterpret_cast<uint4*>(out + vox * outC);
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    uint4 o;
                    __nv_bfloat162* ob = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj)
                        ob[jj] = __floats2bfloat162_rn(v[q * 8 + 2 * jj], v[q * 8 + 2 * jj + 1]);
                    op[q] = o;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tc_tmem_free(tmem, kTcTmemCols);
    }
}

}  // namespace ewg
