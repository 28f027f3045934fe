// Block ILU(0) in the box-8-colour order, and the solver storage order it needs.
//
// Ordering. The grid is cut into 2x2x2 boxes. A box's colour is bit 1 of its cell coordinates
// (i, j, k) -- colour = ((i >> 1) & 1) | ((j >> 1) & 1) << 1 | ((k >> 1) & 1) << 2 -- so two boxes
// of one colour never share a face. The ILU order is colour-major; inside a box the cells follow
// the natural order q = (i & 1) | (j & 1) << 1 | (k & 1) << 2 (x fastest). Boxes of one colour are
// independent, so a colour's boxes are factorized and swept in parallel: the factorization by one
// thread per box that walks its eight cells in order, the sweeps by one warp per place. The factorization is dune-istl's bilu0_decomposition and the
// sweeps its bilu_backsolve on the matrix permuted to this order (the oracle's ORC_ORDER_BOX8
// runs exactly that on the CPU). On the 3D lens problem this order needs about a third fewer
// BiCGStab iterations than the red-black order (64x64x32: 658 against 998 in the first step;
// the reference's natural order takes 583) while every phase stays fully parallel.
//
// Because the grid graph is bipartite, no neighbour of a cell is a neighbour of another
// neighbour, so ILU(0) modifies only diagonal blocks: with D' the pivots,
//   L_ck = A_ck inv(D'_k) for the earlier neighbours k of c,  D'_c = A_cc - sum_k L_ck A_kc,
//   forward   w_c = d_c - sum_{k earlier} L_ck w_k       (colours 0..7, cells q = 0..7)
//   backward  y_c = inv(D'_c) (w_c - sum_{k later} A_ck y_k)   (colours 7..0, q = 7..0)
// and the result is relax * y, as SeqILU applies its relaxation.
//
// Storage ("box-8 order", 3D grids with nx, ny, nz multiples of 4). The N cells fall into 64
// groups by (i mod 4, j mod 4, k mod 4), group g = colour << 3 | q, each a regular lattice with one
// cell per 4x4x4 superblock b = (i >> 2) + nbx ((j >> 2) + nby (k >> 2)). A cell lives at
// g Nb + b (Nb = N / 64). For a fixed (colour, q) the threads of a warp hold consecutive b, so
// every matrix plane and vector access of the sweeps and of the SpMV is coalesced. Matrices keep
// the band-major layout of the linearizer (plane band * 4 + entry) over this cell order.
//
// Neighbours. Across face (axis, side) a cell with box bit c = colour bit and place bit q of the
// axis has, for side -: q = 1: the same box, place q - 1 (earlier); q = 0, c = 1: the box of
// colour c - 1 in the same superblock (earlier); q = 0, c = 0: the box of the superblock before
// (later, absent on the boundary). For side +: q = 0: the same box (later); q = 1, c = 0: the box
// of colour c + 1 in the same superblock (later); q = 1, c = 1: the superblock after (earlier,
// absent on the boundary). For a phase (colour fixed) and a place q all of this is compile-time.
#pragma once

#include "ewg_krylov.cuh"

// Resident blocks per SM the sweep kernels are compiled for (register budget 65536 / (256 x this)).
#ifndef EWG_B8_SWEEP_BLOCKS
#define EWG_B8_SWEEP_BLOCKS 4
#endif
// ... for FP32 matrices, whose blocks take half the registers
#ifndef EWG_B8_SWEEP_BLOCKS_F32
#define EWG_B8_SWEEP_BLOCKS_F32 6
#endif
#define EWG_B8_SWEEP_MINB(TM) (sizeof(TM) == 4 ? EWG_B8_SWEEP_BLOCKS_F32 : EWG_B8_SWEEP_BLOCKS)

namespace ewg {

// The box-8 copies of the matrix (A8, 7 bands), its L factors (L8, 6 bands), inverted pivots and
// E = A_cc - D' (1 band each) are solver-internal and block-packed: the 2x2 block of band b of the
// cell at box-8 position s is the four consecutive values at element offset 4 (b N + s), so a
// block is one 16-byte load in FP32 and two in FP64 (the linearizer's planes keep one entry per
// plane).
template <typename T>
__device__ __forceinline__ void load_pb(const T* __restrict__ A, int64_t N, int band, int64_t s, double b[4]);
template <>
__device__ __forceinline__ void load_pb<float>(const float* __restrict__ A, int64_t N, int band, int64_t s, double b[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(A) + ((int64_t)band * N + s));
    b[0] = v.x; b[1] = v.y; b[2] = v.z; b[3] = v.w;
}
template <>
__device__ __forceinline__ void load_pb<double>(const double* __restrict__ A, int64_t N, int band, int64_t s, double b[4]) {
    const double2* p = reinterpret_cast<const double2*>(A) + 2 * ((int64_t)band * N + s);
    const double2 v0 = __ldg(p), v1 = __ldg(p + 1);
    b[0] = v0.x; b[1] = v0.y; b[2] = v1.x; b[3] = v1.y;
}
// the FP32 blocks kept as FP32 in registers (converted exactly where they are used)
__device__ __forceinline__ void load_pb(const float* __restrict__ A, int64_t N, int band, int64_t s, float b[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(A) + ((int64_t)band * N + s));
    b[0] = v.x; b[1] = v.y; b[2] = v.z; b[3] = v.w;
}
__device__ __forceinline__ void store_pb(float* __restrict__ A, int64_t N, int band, int64_t s, const double b[4]) {
    reinterpret_cast<float4*>(A)[(int64_t)band * N + s] = make_float4((float)b[0], (float)b[1], (float)b[2], (float)b[3]);
}
__device__ __forceinline__ void store_pb(double* __restrict__ A, int64_t N, int band, int64_t s, const double b[4]) {
    double2* p = reinterpret_cast<double2*>(A) + 2 * ((int64_t)band * N + s);
    p[0] = make_double2(b[0], b[1]);
    p[1] = make_double2(b[2], b[3]);
}

struct Box8Pos {
    int bx, by, bz;
};

__device__ __forceinline__ Box8Pos b8_box(const Phys& P, uint32_t b) {
    Box8Pos r;
    const uint32_t row = fastdiv(P.fdNbx, b);
    r.bx = (int)(b - row * (uint32_t)P.nbx);
    const uint32_t bz = fastdiv(P.fdNby, row);
    r.by = (int)(row - bz * (uint32_t)P.nby);
    r.bz = (int)bz;
    return r;
}

// position in box-8 order of natural cell (i, j, k)
__host__ __device__ inline int64_t b8_pos_of(const Phys& P, int i, int j, int k) {
    const int colour = ((i >> 1) & 1) | (((j >> 1) & 1) << 1) | (((k >> 1) & 1) << 2);
    const int q = (i & 1) | ((j & 1) << 1) | ((k & 1) << 2);
    const int64_t b = (int64_t)(i >> 2) + (int64_t)P.nbx * ((j >> 2) + (int64_t)P.nby * (k >> 2));
    return (int64_t)(colour * 8 + q) * P.Nb + b;
}

// Neighbour of the cell (colour C, place Q, superblock b at bp) across face (AXIS, SIDE):
// its group and superblock, whether it exists, and whether it comes earlier in the ILU order.
template <int C, int Q, int AXIS, int SIDE>
struct B8Nbr {
    static constexpr int bit = 1 << AXIS;
    static constexpr bool qa = (Q >> AXIS) & 1;
    static constexpr bool ca = (C >> AXIS) & 1;
    static constexpr bool inBox = SIDE == 0 ? qa : !qa;
    static constexpr bool earlier = SIDE == 0 ? (qa || ca) : (qa && ca);
    // crosses into the neighbouring superblock
    static constexpr bool crosses = SIDE == 0 ? (!qa && !ca) : (qa && ca);
    static constexpr int nC = inBox ? C : (SIDE == 0 ? (qa ? C : (ca ? (C & ~bit) : (C | bit)))
                                                   : (!qa ? C : (!ca ? (C | bit) : (C & ~bit))));
    static constexpr int nQ = inBox ? (Q ^ bit) : (SIDE == 0 ? (Q | bit) : (Q & ~bit));
    static constexpr int group = nC * 8 + nQ;
};

// The faces of a cell of (C, Q) sorted by the ILU position of the neighbour across them:
// neighbours of other colours come in colour order, those in the same box in place order, so the
// key group = colour * 8 + place orders them (the six groups are distinct). The factorization and
// the forward sweep visit faces in ascending order, the backward sweep in descending order, as
// bilu0_decomposition and bilu_backsolve visit the columns of a permuted row.
template <int C, int Q>
struct B8FaceOrder {
    __host__ __device__ static constexpr int group(int dir) {
        const int axis = dir >> 1, side = dir & 1, bit = 1 << axis;
        const bool qa = (Q >> axis) & 1, ca = (C >> axis) & 1;
        const bool inBox = side == 0 ? qa : !qa;
        const int nC = inBox ? C : (side == 0 ? (ca ? (C & ~bit) : (C | bit)) : (!ca ? (C | bit) : (C & ~bit)));
        const int nQ = inBox ? (Q ^ bit) : (side == 0 ? (Q | bit) : (Q & ~bit));
        return nC * 8 + nQ;
    }
    // direction (2 * axis + side) of rank r in ascending neighbour order
    __host__ __device__ static constexpr int dir(int r) {
        for (int d = 0; d < 6; ++d) {
            int rank = 0;
            for (int e = 0; e < 6; ++e) rank += group(e) < group(d) ? 1 : 0;
            if (rank == r) return d;
        }
        return -1;
    }
};

template <int AXIS>
__device__ __forceinline__ int64_t b8_stride(const Phys& P) {
    return AXIS == 0 ? 1 : (AXIS == 1 ? (int64_t)P.nbx : (int64_t)P.nbx * P.nby);
}
template <int AXIS>
__device__ __forceinline__ int b8_coord(const Box8Pos& bp) {
    return AXIS == 0 ? bp.bx : (AXIS == 1 ? bp.by : bp.bz);
}
template <int AXIS>
__device__ __forceinline__ int b8_extent(const Phys& P) {
    return AXIS == 0 ? P.nbx : (AXIS == 1 ? P.nby : P.nbz);
}

// position of the neighbour (or -1) for a compile-time neighbour descriptor
template <int C, int Q, int AXIS, int SIDE>
__device__ __forceinline__ int64_t b8_nbr_pos(const Phys& P, int64_t b, const Box8Pos& bp) {
    using NB = B8Nbr<C, Q, AXIS, SIDE>;
    if (NB::crosses) {
        if (SIDE == 0 && b8_coord<AXIS>(bp) == 0) return -1;
        if (SIDE == 1 && b8_coord<AXIS>(bp) == b8_extent<AXIS>(P) - 1) return -1;
        return (int64_t)NB::group * P.Nb + b + (SIDE == 0 ? -b8_stride<AXIS>(P) : b8_stride<AXIS>(P));
    }
    return (int64_t)NB::group * P.Nb + b;
}

// ---- factorization: one colour, one thread per box ----------------------------------------------

template <typename TM, int C, int Q, int AXIS, int SIDE>
__device__ __forceinline__ void b8_factor_face(const Phys& P, const TM* __restrict__ A, const TM* __restrict__ Dinv,
                                               TM* __restrict__ L, int64_t b, const Box8Pos& bp, int64_t pos,
                                               const double (&dinvBox)[8][4], double D[4]) {
    using NB = B8Nbr<C, Q, AXIS, SIDE>;
    if (!NB::earlier) return;
    const int64_t n = b8_nbr_pos<C, Q, AXIS, SIDE>(P, b, bp);
    if (n < 0) return;
    const int band = band_of(AXIS, SIDE);
    double Ack[4], Dk[4], Akc[4], Lb[4], B[4];
    load_pb(A, P.N, band, pos, Ack);
    if (NB::inBox) {
#pragma unroll
        for (int t = 0; t < 4; ++t) Dk[t] = dinvBox[NB::nQ][t];
    } else {
        load_pb(Dinv, P.N, 0, n, Dk);
    }
    mul2(Ack, Dk, Lb);
    load_pb(A, P.N, opposite_band(band), n, Akc);
    mul2(Lb, Akc, B);
#pragma unroll
    for (int t = 0; t < 4; ++t) D[t] -= B[t];
    store_pb(L, P.N, band - 1, pos, Lb);
}

template <typename TM, int C, int Q>
__device__ __forceinline__ bool b8_factor_cell(const Phys& P, const TM* __restrict__ A, TM* __restrict__ Dinv,
                                               TM* __restrict__ L, TM* __restrict__ E, int64_t b, const Box8Pos& bp,
                                               double (&dinvBox)[8][4]) {
    const int64_t pos = (int64_t)(C * 8 + Q) * P.Nb + b;
    double D[4];
    load_pb(A, P.N, 0, pos, D);
    // every earlier neighbour updates only D (no two neighbours are adjacent), in ascending
    // column order of the permuted row, as bilu0_decomposition's k loop
    using O = B8FaceOrder<C, Q>;
    b8_factor_face<TM, C, Q, (O::dir(0) >> 1), (O::dir(0) & 1)>(P, A, Dinv, L, b, bp, pos, dinvBox, D);
    b8_factor_face<TM, C, Q, (O::dir(1) >> 1), (O::dir(1) & 1)>(P, A, Dinv, L, b, bp, pos, dinvBox, D);
    b8_factor_face<TM, C, Q, (O::dir(2) >> 1), (O::dir(2) & 1)>(P, A, Dinv, L, b, bp, pos, dinvBox, D);
    b8_factor_face<TM, C, Q, (O::dir(3) >> 1), (O::dir(3) & 1)>(P, A, Dinv, L, b, bp, pos, dinvBox, D);
    b8_factor_face<TM, C, Q, (O::dir(4) >> 1), (O::dir(4) & 1)>(P, A, Dinv, L, b, bp, pos, dinvBox, D);
    b8_factor_face<TM, C, Q, (O::dir(5) >> 1), (O::dir(5) & 1)>(P, A, Dinv, L, b, bp, pos, dinvBox, D);
    // E = A_cc - D' (what the pivot lost to the earlier neighbours), for the preconditioned SpMV
    double Ad[4], Ec[4];
    load_pb(A, P.N, 0, pos, Ad);
#pragma unroll
    for (int t = 0; t < 4; ++t) Ec[t] = Ad[t] - D[t];
    store_pb(E, P.N, 0, pos, Ec);
    double o[4];
    const bool ok = inv2(D, o);
    if (!ok) o[0] = o[1] = o[2] = o[3] = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) dinvBox[Q][t] = o[t];
    store_pb(Dinv, P.N, 0, pos, o);
    return ok;
}

// Colour levels. Adjacent boxes differ in exactly one colour bit, so boxes whose colours have the
// same number of set bits never share a face: colours 1, 2, 4 depend only on colour 0 and colours
// 3, 5, 6 only on 1, 2, 4. A phase of the factorization or the sweeps can therefore run one launch
// per level -- {0}, {1, 2, 4}, {3, 5, 6}, {7} (the backward sweep in the reverse order) -- with the
// same results as one launch per colour in colour order: a cell's values depend only on its
// finished neighbours, and the terms of its row are summed in the same order. The batched ensemble
// does (its launches are the cost there); the single problem keeps one launch per colour.
template <int LEVEL>
struct B8Level {
    static constexpr int count = (LEVEL == 0 || LEVEL == 3) ? 1 : 3;
    __host__ __device__ static constexpr int colour(int i) {
        return LEVEL == 0 ? 0 : (LEVEL == 3 ? 7 : (LEVEL == 1 ? (1 << i) : (7 ^ (1 << i))));
    }
};
// calls F::template run<C>() for colour i of the level (i uniform over the block)
#define EWG_B8_LEVEL_DISPATCH(LEVEL, i, CALL)                              \
    do {                                                                   \
        if (B8Level<LEVEL>::count == 1) { CALL(B8Level<LEVEL>::colour(0)); } \
        else if ((i) == 0) { CALL(B8Level<LEVEL>::colour(0)); }            \
        else if ((i) == 1) { CALL(B8Level<LEVEL>::colour(1)); }            \
        else { CALL(B8Level<LEVEL>::colour(2)); }                          \
    } while (0)

template <typename TM, int C>
__device__ __forceinline__ bool b8_factor_box(const Phys& P, const TM* __restrict__ A, TM* __restrict__ Dinv,
                                              TM* __restrict__ L, TM* __restrict__ E, int64_t b) {
    const Box8Pos bp = b8_box(P, (uint32_t)b);
    double dinvBox[8][4];
    bool ok = true;
    ok &= b8_factor_cell<TM, C, 0>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 1>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 2>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 3>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 4>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 5>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 6>(P, A, Dinv, L, E, b, bp, dinvBox);
    ok &= b8_factor_cell<TM, C, 7>(P, A, Dinv, L, E, b, bp, dinvBox);
    return ok;
}

// factorization of colour C: one thread per box
template <typename TM, int C>
__global__ void __launch_bounds__(kSolBlock) k_b8_factor(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                          TM* __restrict__ Dinv, TM* __restrict__ L, TM* __restrict__ E,
                                                          int* bad) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < P.Nb; b += (int64_t)gridDim.x * blockDim.x)
        if (!b8_factor_box<TM, C>(P, A, Dinv, L, E, b)) atomicOr(bad, 1);
}

// ---- sweeps: one warp per place, one lane per box ---------------------------------------------------
//
// A block of kB8Block threads takes 32 consecutive superblocks b0 .. b0 + 31 of one colour: warp q
// holds place q of the 32 boxes, lane l the box of superblock b0 + l, so every load and store of a
// warp touches 32 consecutive positions of one group. Inside a box the dependencies of the sweeps
// form the 3-cube of the places (a place depends on the places that differ from it in one bit and
// come earlier), so the eight places run in four levels -- forward by the number of set bits of q,
// backward by the number of clear bits -- with the box's finished values passed through shared
// memory and one block barrier between levels. Every load of a cell (its vector entry, the blocks
// and the other colours' values) is issued before the levels; a level only adds the terms of the
// same box.
//
// Summation order. In ascending ILU order the neighbours of a cell are: the boxes of earlier
// colours, then the cells of the same box by place, then the boxes of later colours (the key
// group = colour * 8 + place, B8FaceOrder). The forward sweep subtracts its terms in ascending
// order and the backward sweep in descending order, so the terms of other boxes come first in
// both and the terms of the same box last -- exactly the split into "before the levels" and "in a
// level", which keeps each cell's sums in bilu_backsolve's column order.

constexpr int kB8Block = 256;  // 8 places x 32 boxes

// Inside a box each cell has one neighbour per axis (place bit flipped): an earlier one where the
// place bit is set, a later one where it is clear. The blocks of these faces are indexed by axis.

// forward, before the levels: the terms of earlier colours, and the blocks of the same box
template <typename TM, typename TV, int C, int Q, int R>
__device__ __forceinline__ void b8_fwd_far(const Phys& P, const TM* __restrict__ L,
                                           const typename V2T<TV>::type* __restrict__ w, int64_t b, const Box8Pos& bp,
                                           int64_t pos, double& r0, double& r1, TM (&Lin)[3][4]) {
    using O = B8FaceOrder<C, Q>;
    constexpr int dir = O::dir(R), AXIS = dir >> 1, SIDE = dir & 1;
    using NB = B8Nbr<C, Q, AXIS, SIDE>;
    if (!NB::earlier) return;
    if (NB::inBox) {
        load_pb(L, P.N, band_of(AXIS, SIDE) - 1, pos, Lin[AXIS]);
        return;
    }
    const int64_t n = b8_nbr_pos<C, Q, AXIS, SIDE>(P, b, bp);
    if (n < 0) return;
    double Lb[4];
    load_pb(L, P.N, band_of(AXIS, SIDE) - 1, pos, Lb);
    const auto wk = w[n];
    const double x0 = (double)wk.x, x1 = (double)wk.y;
    r0 -= Lb[0] * x0; r0 -= Lb[1] * x1;
    r1 -= Lb[2] * x0; r1 -= Lb[3] * x1;
}

template <typename TM, typename TV, int C, int Q>
__device__ __forceinline__ void b8_fwd_far_all(const Phys& P, const TM* __restrict__ L,
                                               const typename V2T<TV>::type* __restrict__ w, int64_t b, int64_t pos,
                                               double& r0, double& r1, TM (&Lin)[3][4]) {
    const Box8Pos bp = b8_box(P, (uint32_t)b);
    b8_fwd_far<TM, TV, C, Q, 0>(P, L, w, b, bp, pos, r0, r1, Lin);
    b8_fwd_far<TM, TV, C, Q, 1>(P, L, w, b, bp, pos, r0, r1, Lin);
    b8_fwd_far<TM, TV, C, Q, 2>(P, L, w, b, bp, pos, r0, r1, Lin);
    b8_fwd_far<TM, TV, C, Q, 3>(P, L, w, b, bp, pos, r0, r1, Lin);
    b8_fwd_far<TM, TV, C, Q, 4>(P, L, w, b, bp, pos, r0, r1, Lin);
    b8_fwd_far<TM, TV, C, Q, 5>(P, L, w, b, bp, pos, r0, r1, Lin);
}

// forward, in its level: the terms of the same box, ascending
template <int C, int Q, int R, typename MT>
__device__ __forceinline__ void b8_fwd_near(const double2 (&S)[8][32], int lane, const MT (&Lin)[3][4], double& r0,
                                            double& r1) {
    using O = B8FaceOrder<C, Q>;
    constexpr int dir = O::dir(R), AXIS = dir >> 1, SIDE = dir & 1;
    using NB = B8Nbr<C, Q, AXIS, SIDE>;
    if (!NB::earlier || !NB::inBox) return;
    const double2 v = S[NB::nQ][lane];
    r0 -= Lin[AXIS][0] * v.x; r0 -= Lin[AXIS][1] * v.y;
    r1 -= Lin[AXIS][2] * v.x; r1 -= Lin[AXIS][3] * v.y;
}

template <int C, int Q, typename MT>
__device__ __forceinline__ void b8_fwd_near_all(const double2 (&S)[8][32], int lane, const MT (&Lin)[3][4],
                                                double& r0, double& r1) {
    b8_fwd_near<C, Q, 0>(S, lane, Lin, r0, r1);
    b8_fwd_near<C, Q, 1>(S, lane, Lin, r0, r1);
    b8_fwd_near<C, Q, 2>(S, lane, Lin, r0, r1);
    b8_fwd_near<C, Q, 3>(S, lane, Lin, r0, r1);
    b8_fwd_near<C, Q, 4>(S, lane, Lin, r0, r1);
    b8_fwd_near<C, Q, 5>(S, lane, Lin, r0, r1);
}

#define EWG_B8_PLACE_SWITCH(q, CALL) \
    switch (q) {                     \
    case 0: CALL(0); break;          \
    case 1: CALL(1); break;          \
    case 2: CALL(2); break;          \
    case 3: CALL(3); break;          \
    case 4: CALL(4); break;          \
    case 5: CALL(5); break;          \
    case 6: CALL(6); break;          \
    default: CALL(7); break;         \
    }

// Forward sweep of colour C over the 32 boxes of superblocks b0 .. b0 + 31 (boxes past P.Nb are
// idle): warp q = place q, lane = box. Every thread of the block calls it; S holds the box values.
template <typename TM, typename TV, int C>
__device__ __forceinline__ void b8_forward_tile(const Phys& P, const TM* __restrict__ L,
                                                const typename V2T<TV>::type* __restrict__ d,
                                                typename V2T<TV>::type* __restrict__ w, int64_t b0,
                                                double2 (&S)[8][32], int lane, int q) {
    const int level = __popc(q);
    const int64_t b = b0 + lane;
    const bool valid = b < P.Nb;
    const int64_t pos = (int64_t)(C * 8 + q) * P.Nb + b;
    double r0 = 0.0, r1 = 0.0;
    TM Lin[3][4];
    if (valid) {
        const auto ds = d[pos];
        r0 = (double)ds.x;
        r1 = (double)ds.y;
#define EWG_B8_CALL(Q) b8_fwd_far_all<TM, TV, C, Q>(P, L, w, b, pos, r0, r1, Lin)
        EWG_B8_PLACE_SWITCH(q, EWG_B8_CALL)
#undef EWG_B8_CALL
    }
#pragma unroll
    for (int lev = 0; lev < 4; ++lev) {
        if (lev > 0) __syncthreads();
        if (lev == level) {
#define EWG_B8_CALL(Q) b8_fwd_near_all<C, Q>(S, lane, Lin, r0, r1)
            EWG_B8_PLACE_SWITCH(q, EWG_B8_CALL)
#undef EWG_B8_CALL
            typename V2T<TV>::type o;
            o.x = (TV)r0;
            o.y = (TV)r1;
            if (valid) w[pos] = o;
            // later places read the stored (rounded) value, as the reference's vector holds it
            S[q][lane] = make_double2((double)o.x, (double)o.y);
        }
    }
}

// forward sweep of colour C: w_c = d_c - sum_{k earlier} L_ck w_k. (One launch per colour: a
// launch per colour level, with the three colours' code in one kernel, ran 10 % slower here.)
template <typename TM, typename TV, int C>
__global__ void __launch_bounds__(kB8Block, EWG_B8_SWEEP_MINB(TM)) k_b8_forward(const __grid_constant__ Phys P, const TM* __restrict__ L,
                                                           const typename V2T<TV>::type* __restrict__ d,
                                                           typename V2T<TV>::type* __restrict__ w,
                                                           const int* __restrict__ status) {
    pdl_enter();
    if (status && *status != ST_RUNNING) return;  // uniform over the grid
    __shared__ double2 SB[2][8][32];  // two tiles' box values (a tile's levels order its own)
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    const int64_t nTiles = (P.Nb + 31) >> 5;
    int k = 0;
    // no barrier between tiles: the next tile writes the other buffer, and the tile after it can
    // only start once every warp has passed the next tile's first level barrier
    for (int64_t tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++k)
        b8_forward_tile<TM, TV, C>(P, L, d, w, tile * 32, SB[k & 1], lane, q);
}

// backward, before the levels: the terms of later colours, and the blocks of the same box
template <typename TM, typename TV, int C, int Q, int R>
__device__ __forceinline__ void b8_bwd_far(const Phys& P, const TM* __restrict__ A,
                                           const typename V2T<TV>::type* __restrict__ y, int64_t b, const Box8Pos& bp,
                                           int64_t pos, double winv, double& r0, double& r1, TM (&Ain)[3][4]) {
    using O = B8FaceOrder<C, Q>;
    constexpr int dir = O::dir(R), AXIS = dir >> 1, SIDE = dir & 1;
    using NB = B8Nbr<C, Q, AXIS, SIDE>;
    if (NB::earlier) return;
    if (NB::inBox) {
        load_pb(A, P.N, band_of(AXIS, SIDE), pos, Ain[AXIS]);
        return;
    }
    const int64_t n = b8_nbr_pos<C, Q, AXIS, SIDE>(P, b, bp);
    if (n < 0) return;
    double Ab[4];
    load_pb(A, P.N, band_of(AXIS, SIDE), pos, Ab);
    const auto yk = y[n];
    double x0 = (double)yk.x, x1 = (double)yk.y;
    if (winv != 1.0) { x0 *= winv; x1 *= winv; }
    r0 -= Ab[0] * x0; r0 -= Ab[1] * x1;
    r1 -= Ab[2] * x0; r1 -= Ab[3] * x1;
}

// descending columns, as bilu_backsolve's backward loop
template <typename TM, typename TV, int C, int Q>
__device__ __forceinline__ void b8_bwd_far_all(const Phys& P, const TM* __restrict__ A,
                                               const typename V2T<TV>::type* __restrict__ y, int64_t b, int64_t pos,
                                               double winv, double& r0, double& r1, TM (&Ain)[3][4]) {
    const Box8Pos bp = b8_box(P, (uint32_t)b);
    b8_bwd_far<TM, TV, C, Q, 5>(P, A, y, b, bp, pos, winv, r0, r1, Ain);
    b8_bwd_far<TM, TV, C, Q, 4>(P, A, y, b, bp, pos, winv, r0, r1, Ain);
    b8_bwd_far<TM, TV, C, Q, 3>(P, A, y, b, bp, pos, winv, r0, r1, Ain);
    b8_bwd_far<TM, TV, C, Q, 2>(P, A, y, b, bp, pos, winv, r0, r1, Ain);
    b8_bwd_far<TM, TV, C, Q, 1>(P, A, y, b, bp, pos, winv, r0, r1, Ain);
    b8_bwd_far<TM, TV, C, Q, 0>(P, A, y, b, bp, pos, winv, r0, r1, Ain);
}

template <int C, int Q, int R, typename MT>
__device__ __forceinline__ void b8_bwd_near(const double2 (&S)[8][32], int lane, const MT (&Ain)[3][4], double& r0,
                                            double& r1) {
    using O = B8FaceOrder<C, Q>;
    constexpr int dir = O::dir(R), AXIS = dir >> 1, SIDE = dir & 1;
    using NB = B8Nbr<C, Q, AXIS, SIDE>;
    if (NB::earlier || !NB::inBox) return;
    const double2 v = S[NB::nQ][lane];
    r0 -= Ain[AXIS][0] * v.x; r0 -= Ain[AXIS][1] * v.y;
    r1 -= Ain[AXIS][2] * v.x; r1 -= Ain[AXIS][3] * v.y;
}

template <int C, int Q, typename MT>
__device__ __forceinline__ void b8_bwd_near_all(const double2 (&S)[8][32], int lane, const MT (&Ain)[3][4],
                                                double& r0, double& r1) {
    b8_bwd_near<C, Q, 5>(S, lane, Ain, r0, r1);
    b8_bwd_near<C, Q, 4>(S, lane, Ain, r0, r1);
    b8_bwd_near<C, Q, 3>(S, lane, Ain, r0, r1);
    b8_bwd_near<C, Q, 2>(S, lane, Ain, r0, r1);
    b8_bwd_near<C, Q, 1>(S, lane, Ain, r0, r1);
    b8_bwd_near<C, Q, 0>(S, lane, Ain, r0, r1);
}

// Backward sweep of colour C over the 32 boxes of superblocks b0 .. b0 + 31 (as b8_forward_tile).
template <typename TM, typename TV, int C>
__device__ __forceinline__ void b8_backward_tile(const Phys& P, const TM* __restrict__ A, const TM* __restrict__ Dinv,
                                                 const typename V2T<TV>::type* __restrict__ wv,
                                                 typename V2T<TV>::type* __restrict__ y, double w, double winv,
                                                 int64_t b0, double2 (&S)[8][32], int lane, int q) {
    const int level = 3 - __popc(q);
    const int64_t b = b0 + lane;
    const bool valid = b < P.Nb;
    const int64_t pos = (int64_t)(C * 8 + q) * P.Nb + b;
    double r0 = 0.0, r1 = 0.0;
    TM Ain[3][4], Di[4] = {(TM)0, (TM)0, (TM)0, (TM)0};
    if (valid) {
        const auto ws = wv[pos];
        r0 = (double)ws.x;
        r1 = (double)ws.y;
#define EWG_B8_CALL(Q) b8_bwd_far_all<TM, TV, C, Q>(P, A, y, b, pos, winv, r0, r1, Ain)
        EWG_B8_PLACE_SWITCH(q, EWG_B8_CALL)
#undef EWG_B8_CALL
        load_pb(Dinv, P.N, 0, pos, Di);
    }
#pragma unroll
    for (int lev = 0; lev < 4; ++lev) {
        if (lev > 0) __syncthreads();
        if (lev == level) {
#define EWG_B8_CALL(Q) b8_bwd_near_all<C, Q>(S, lane, Ain, r0, r1)
            EWG_B8_PLACE_SWITCH(q, EWG_B8_CALL)
#undef EWG_B8_CALL
            const double u0 = Di[0] * r0 + Di[1] * r1, u1 = Di[2] * r0 + Di[3] * r1;
            typename V2T<TV>::type o;
            o.x = (TV)(w * u0);
            o.y = (TV)(w * u1);
            if (valid) y[pos] = o;
            // the unscaled value as a later-colour reader recovers it from the stored one
            if (w == 1.0) S[q][lane] = make_double2((double)o.x, (double)o.y);
            else S[q][lane] = make_double2((double)o.x * winv, (double)o.y * winv);
        }
    }
}

// backward sweep of colour C: y_c = inv(D'_c) (w_c - sum_{k later} A_ck y_k), output relax * y.
// w stays in its own vector (the preconditioned SpMV reads it again). The stored outputs of later
// colours are relax * y; the coupling term works on unscaled y, as the reference's backward solve
// runs before its final scaling.
template <typename TM, typename TV, int C>
__global__ void __launch_bounds__(kB8Block, EWG_B8_SWEEP_MINB(TM)) k_b8_backward(const __grid_constant__ Phys P, const TM* __restrict__ A,
                                                            const TM* __restrict__ Dinv,
                                                            const typename V2T<TV>::type* __restrict__ wv,
                                                            typename V2T<TV>::type* __restrict__ y,
                                                            const int* __restrict__ status, double w) {
    pdl_enter();
    if (status && *status != ST_RUNNING) return;  // uniform over the grid
    __shared__ double2 SB[2][8][32];
    const double winv = 1.0 / w;
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    const int64_t nTiles = (P.Nb + 31) >> 5;
    int k = 0;
    for (int64_t tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++k)
        b8_backward_tile<TM, TV, C>(P, A, Dinv, wv, y, w, winv, tile * 32, SB[k & 1], lane, q);
}

#undef EWG_B8_PLACE_SWITCH

// ---- SpMV row in box-8 order ---------------------------------------------------------------------
//
// With g = colour << 3 | place, the group of the neighbour across (axis, side) flips the place bit
// of the axis (same box) or both the place and the colour bit (other box): side -: same box iff the
// place bit is set; side +: same box iff it is clear. The neighbour lies in the superblock before
// (side -, place and colour bits clear) or after (side +, both set), else in the same superblock.
// All of this is uniform over a warp when N / 64 is a multiple of 32 (groups are contiguous).

struct B8Step {
    int pos;      // neighbour position, or the cell itself when there is no neighbour
    bool exists;
};

__device__ __forceinline__ B8Step b8_step(const Phys& P, int g, int b, const Box8Pos& bp, int axis, int side) {
    const int bit = 1 << axis;
    const bool qa = (g >> axis) & 1, ca = (g >> (3 + axis)) & 1;
    const bool sameBox = side == 0 ? qa : !qa;
    const int gN = sameBox ? (g ^ bit) : (g ^ (bit << 3) ^ bit);
    const bool prev = side == 0 && !qa && !ca, next = side == 1 && qa && ca;
    const int coord = axis == 0 ? bp.bx : (axis == 1 ? bp.by : bp.bz);
    const int ext = axis == 0 ? P.nbx : (axis == 1 ? P.nby : P.nbz);
    const int stride = axis == 0 ? 1 : (axis == 1 ? P.nbx : P.nbx * P.nby);
    B8Step r;
    r.exists = !(prev && coord == 0) && !(next && coord == ext - 1);
    const int delta = prev ? -stride : (next ? stride : 0);
    r.pos = r.exists ? gN * (int)P.Nb + b + delta : g * (int)P.Nb + b;
    return r;
}

// y_s = sum over the row's blocks in ascending natural column order (-z -y -x diag +x +y +z), the
// order of the reference's BCRS mv. Blocks of missing neighbours are zero in the band storage, so
// every band is read; the vector entry of a missing neighbour is taken as zero.
template <typename TM, typename TV>
__device__ __forceinline__ void spmv_row_b8(const Phys& P, const TM* __restrict__ A,
                                            const typename V2T<TV>::type* __restrict__ x, int64_t s64,
                                            double& a0, double& a1) {
    const int s = (int)s64;  // N < 2^31
    const int g = (int)fastdiv(P.fdNb, (uint32_t)s);
    const int b = s - g * (int)P.Nb;
    const Box8Pos bp = b8_box(P, (uint32_t)b);
    const int bands[7] = {5, 3, 1, 0, 2, 4, 6};
    a0 = 0.0;
    a1 = 0.0;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const int band = bands[q];
        double B[4];
        load_pb(A, P.N, band, s, B);
        double x0 = 0.0, x1 = 0.0;
        if (band == 0) {
            const auto xk = x[s];
            x0 = (double)xk.x;
            x1 = (double)xk.y;
        } else {
            const B8Step st = b8_step(P, g, b, bp, (band - 1) >> 1, (band - 1) & 1);
            const auto xk = x[st.pos];
            if (st.exists) {
                x0 = (double)xk.x;
                x1 = (double)xk.y;
            }
        }
        a0 += B[0] * x0; a0 += B[1] * x1;
        a1 += B[2] * x0; a1 += B[3] * x1;
    }
}

// v = A y for y = relax M^-1 d, from the sweeps' intermediate w = (D' + L_A)^-1 d: the backward
// sweep gave D' (y / relax) = w - U_A (y / relax), so
//   A y = L_A y + A_cc y + U_A y = L_A y + (A_cc - D') y + relax w,
// with E = A_cc - D' from the factorization. The blocks of the later neighbours (U_A, half the
// off-diagonal blocks) are not read. Equal to A y in exact arithmetic; the sums differ in rounding.
template <typename TM, typename TV>
__device__ __forceinline__ void spmv_row_b8_precond(const Phys& P, const TM* __restrict__ A, const TM* __restrict__ E,
                                                    const typename V2T<TV>::type* __restrict__ wv, double relax,
                                                    const typename V2T<TV>::type* __restrict__ y, int64_t s64,
                                                    double& a0, double& a1) {
    const int s = (int)s64;
    const int g = (int)fastdiv(P.fdNb, (uint32_t)s);
    const int b = s - g * (int)P.Nb;
    const Box8Pos bp = b8_box(P, (uint32_t)b);
    const auto wc = wv[s];
    a0 = relax * (double)wc.x;
    a1 = relax * (double)wc.y;
    {
        double B[4];
        load_pb(E, P.N, 0, s, B);
        const auto yc = y[s];
        const double x0 = (double)yc.x, x1 = (double)yc.y;
        a0 += B[0] * x0; a0 += B[1] * x1;
        a1 += B[2] * x0; a1 += B[3] * x1;
    }
    const int bands[6] = {5, 3, 1, 2, 4, 6};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int band = bands[q];
        const int axis = (band - 1) >> 1, side = (band - 1) & 1;
        const bool qa = (g >> axis) & 1, ca = (g >> (3 + axis)) & 1;
        const bool earlier = side == 0 ? (qa || ca) : (qa && ca);
        if (!earlier) continue;  // uniform over a warp
        const B8Step st = b8_step(P, g, b, bp, axis, side);
        if (!st.exists) continue;
        double B[4];
        load_pb(A, P.N, band, s, B);
        const auto yk = y[st.pos];
        const double x0 = (double)yk.x, x1 = (double)yk.y;
        a0 += B[0] * x0; a0 += B[1] * x1;
        a1 += B[2] * x0; a1 += B[3] * x1;
    }
}

// ---- conversion between the split order and box-8 order -------------------------------------------

// box-8 position s -> split-order position of the same cell
__device__ __forceinline__ int64_t b8_to_split_pos(const Phys& P, int64_t s) {
    const uint32_t g = fastdiv(P.fdNb, (uint32_t)s);
    const int64_t b = s - (int64_t)g * P.Nb;
    const int C = (int)(g >> 3), Q = (int)(g & 7);
    const Box8Pos bp = b8_box(P, (uint32_t)b);
    const int i = 4 * bp.bx + 2 * (C & 1) + (Q & 1);
    const int j = 4 * bp.by + 2 * ((C >> 1) & 1) + ((Q >> 1) & 1);
    const int k = 4 * bp.bz + 2 * ((C >> 2) & 1) + ((Q >> 2) & 1);
    const int64_t c = (int64_t)i + (int64_t)P.nx * (j + (int64_t)P.ny * k);
    const int col = (i + j + k) & 1;
    return (int64_t)col * P.Nh + (c >> 1);
}

// matrix planes (nPlanes = 4 x bands planes of N values) into the block-packed box-8 copy:
// out block (band, s8) = in planes (4 band .. 4 band + 3)[split(s8)], converting TI -> TO.
// One thread per pair of cells two apart in x (colour bit 0 clear and set, same place and box):
// they are neighbours in the split order (split positions sp and sp + 1, sp even), so each plane
// is read as one aligned pair and every sector read is used whole; each block is written as one
// 16- or 32-byte packed store.
template <typename TI, typename TO>
__global__ void k_b8_matrix_from_split(const __grid_constant__ Phys P, int nPlanes, const TI* __restrict__ in,
                                       TO* __restrict__ out) {
    using TI2 = typename V2T<TI>::type;
    const TI2* __restrict__ in2 = reinterpret_cast<const TI2*>(in);
    const int64_t half = P.N / 2;
    const int bands = nPlanes / 4;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < half; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gi = t / P.Nb;                            // 32 groups with colour bit 0 clear
        const int64_t b = t - gi * P.Nb;
        const int64_t g = ((gi >> 3) << 4) | (gi & 7);          // colour = g >> 3, place = g & 7
        const int64_t s = g * P.Nb + b, s2 = s + 8 * P.Nb;      // colour bit 0 clear / set
        const int64_t sp = b8_to_split_pos(P, s);              // even; s2 sits at sp + 1
        for (int band = 0; band < bands; ++band) {
            double v[4], w[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const TI2 a = in2[((int64_t)(4 * band + c) * P.N + sp) >> 1];
                v[c] = (double)a.x;
                w[c] = (double)a.y;
            }
            store_pb(out, P.N, band, s, v);
            store_pb(out, P.N, band, s2, w);
        }
    }
}

// vectors: TOB8 = true: out[s8] = in[split(s8)], else out[split(s8)] = in[s8]
template <typename TI, typename TO, bool TOB8>
__global__ void k_b8_vector(const __grid_constant__ Phys P, const typename V2T<TI>::type* __restrict__ in,
                            typename V2T<TO>::type* __restrict__ out) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sp = b8_to_split_pos(P, s);
        const auto v = TOB8 ? in[sp] : in[s];
        typename V2T<TO>::type o;
        o.x = (TO)v.x;
        o.y = (TO)v.y;
        if (TOB8) out[s] = o;
        else out[sp] = o;
    }
}

// ---- host launchers (ewg_box8.cu) -------------------------------------------------------------

// Copy nPlanes planes of N values from the split order into box-8 order.
template <typename TI, typename TO>
void b8_matrix_from_split(ewg_ctx* ctx, int nPlanes, const TI* in, TO* out);
// One vector between the split order and box-8 order (toB8: split -> box-8).
template <typename TI, typename TO, bool TOB8>
void b8_vector(ewg_ctx* ctx, const typename V2T<TI>::type* in, typename V2T<TO>::type* out);
// The eight colour phases of the factorization (L factors, inverted pivots, E = A_cc - D');
// *bad |= 1 on a singular pivot.
template <typename T>
void b8_factor(ewg_ctx* ctx, const T* A8, T* Dinv8, T* L8, T* E8, int* bad);
// y = relax M^-1 d with the forward sweep's intermediate left in w (d, w, y distinct); kernels
// return at once when *status != running.
template <typename T>
void b8_apply(ewg_ctx* ctx, const T* A8, const T* Dinv8, const T* L8, double relax,
              const typename V2T<T>::type* d, typename V2T<T>::type* w, typename V2T<T>::type* y, const int* status);

}  // namespace ewg
