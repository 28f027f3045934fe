// Per-cell pieces of the ECFV + AD linearization shared by the single-problem kernels
// (ewg_linearize.cu) and the batched ensemble (ewg_ensemble.cu).
//
// The element of cell i focuses on its own DOF (fvbaseadlocallinearizer.hh:178-297): it evaluates
// its local residual with derivatives with respect to x_i only, writes its residual row r_i and
// scatters the Jacobian column i, J[i][i] and J[j][i] for every face neighbour j
// (fvbaselinearizer.hh:483-512).
#pragma once

#include "ewg_physics.cuh"

namespace ewg {

// intensive quantities of one cell that its neighbours need (immiscibleintensivequantities.hh
// :87-145): p_c, lambda_w = k_rw / mu_w, lambda_n = k_rn / mu_n, each with d/dS_w
struct IqVals {
    double pc, dpc, lw, dlw, ln, dln;
};
__device__ __forceinline__ IqVals intensive_values_full(const Phys& P, double Sw, int lensFlag) {
    const LawDev& L = P.law[lensFlag];
    MatOut m = material(L, Sw);
    // mobility = kr / mu as an AD quotient with a constant denominator
    const double muw = P.mu[0], mun = P.mu[1];
    IqVals o;
    o.pc = m.pc.v;
    o.dpc = m.pc.d;
    o.lw = m.krw.v / muw;
    o.dlw = (muw * m.krw.d) / (muw * muw);
    o.ln = m.krn.v / mun;
    o.dln = (mun * m.krn.d) / (mun * mun);
    return o;
}
// The same with the state of all cells the DNAPL has not reached, S_w = 1, taken from the values
// intensive_values_full gave for it at context creation (P.sat1): the same bits without the
// material-law evaluation.
__device__ __forceinline__ IqVals intensive_values(const Phys& P, double Sw, int lensFlag) {
    if (Sw == 1.0) {
        const double* c = P.sat1[lensFlag];
        return IqVals{c[0], c[1], c[2], c[3], c[4], c[5]};
    }
    return intensive_values_full(P, Sw, lensFlag);
}

// the same, written to the cache in 6 planes (pc, dpc, lw, dlw, ln, dln); without `deriv` only the
// values a neighbour reads (planes 0, 2, 4), for kernels that evaluate their own cell's quantities
__device__ __forceinline__ void intensive_cell(const Phys& P, const double2* __restrict__ x,
                                               const uint8_t* __restrict__ lens, double* __restrict__ iq,
                                               int64_t s, bool deriv = true) {
    const int64_t N = P.N;
    const IqVals o = intensive_values(P, x[s].y, lens[s]);
    iq[s] = o.pc;
    iq[2 * N + s] = o.lw;
    iq[4 * N + s] = o.ln;
    if (deriv) {
        iq[N + s] = o.dpc;
        iq[3 * N + s] = o.dlw;
        iq[5 * N + s] = o.dln;
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

// One interior face seen from the focus cell i (darcyfluxmodule.hh:185-324, 461-527;
// immisciblelocalresidual.hh:123-149): adds the mass fluxes to R_i and dR_i/dx_i and returns the
// block dR_j/dx_i of the neighbour's local residual (already divided by the neighbour's volume).
template <int AXIS>
__device__ __forceinline__ void interior_face(const Phys& P, int side, int idxA, double Ki, const double pI[2],
                                              double dpcI, const double lam[2], const double dlam[2],
                                              double2 xj, double Kj, double pcj, const double lamj[2],
                                              double R[2], double D[2][2], double Dj[4]) {
    const double h = P.h[AXIS];
    const int ia = idxA + (AXIS == 2 ? P.kOrigin : 0);
    const double xc = (ia + 0.5) * h;
    const double xcj = (ia + (side ? 1 : -1) + 0.5) * h;
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
            const double xf = (ia + side) * h;
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
    for (int d = 0; d < 3; ++d) xc[d] = d < DIM ? (idx[d] + (d == 2 ? P.kOrigin : 0) + 0.5) * P.h[d] : 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) xf[d] = xc[d];
    xf[AXIS] = (idx[AXIS] + (AXIS == 2 ? P.kOrigin : 0) + side) * P.h[AXIS];
    const double area = P.area[AXIS];
    const bool left = xf[0] < 0.0 + P.eps, right = xf[0] > P.L[0] - P.eps;
    if (left || right) {
        const double g1 = -P.g;
        const double depth = P.L[1] - xf[1];
        const double pw = left ? __dsub_rn(P.pRef, P.leftScale * P.rho[0] * g1 * depth)
                               : __dsub_rn(P.pRef, P.rho[0] * g1 * depth);
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
            grad = __dadd_rn(grad, __dmul_rn(distIn, pStatIn / absDistSq));
            const bool upB = grad * nA > 0;
            const double lamU = upB ? P.bndLam[lensI][a] : lam[a];
            const double dlamU = upB ? 0.0 : dlam[a];
            const double sK = Ki * grad;
            const double vel = sK * (-lamU);
            const double dvelP = (Ki * dgP) * (-lamU);
            const double dvelS = __dadd_rn((Ki * dgS) * (-lamU), (-dlamU) * sK);
            R[a] = __dadd_rn(R[a], vel * nA * rho * area);
            D[a][0] = __dadd_rn(D[a][0], dvelP * nA * rho * area);
            D[a][1] = __dadd_rn(D[a][1], dvelS * nA * rho * area);
        }
        return;
    }
    const bool upper = xf[1] > P.L[1] - P.eps;
    bool inlet = upper && xf[0] > P.inletXlo && xf[0] < P.inletXhi;
    if (DIM == 3) inlet = inlet && xf[2] > P.inletZlo && xf[2] < P.inletZhi;
    if (inlet) R[1] = __dadd_rn(R[1], P.inletRate * area);
}

// ---- 3D interior cells --------------------------------------------------------------------------
//
// Every face of an interior cell has a neighbour, so the per-cell work is branch-free: six
// interior faces and the storage term. The face geometry (gradient coefficient and hydrostatic
// correction) comes from a small table instead of being recomputed from cell positions, and the
// scalings by 1/V are multiplications. The two-point gradient is formed with explicitly rounded
// products and sums (no fused multiply-add) so that its sign, which selects the upstream cell,
// is the one an unfused CPU evaluation gets; the sums into the residual and the Jacobian blocks are
// explicitly rounded too, so that every kernel inlining these functions gets the same bits.

template <int AXIS>
__device__ __forceinline__ void interior_face_tab(const Phys& P, const FaceGeo& G, int side, double Ki,
                                                  const double pI[2], double dpcI, const double lam[2],
                                                  const double dlam[2], double pwj, double Kj, double pcj,
                                                  double lwj, double lnj, double R[2], double D[2][2],
                                                  double Dj[4]) {
    const double coef = G.coef;
    const double Kf = harmonic_mean(Ki, Kj);
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const double pJ = a == 0 ? pwj : pwj + (pcj - 0.0);
        const double deltay = pJ - pI[a];
        double grad = __dmul_rn(deltay, coef);
        const double dgP = -coef;
        const double dgS = a == 0 ? 0.0 : -dpcI * coef;
        if (AXIS == 1) grad = __dadd_rn(grad, __dmul_rn(G.dA, G.gt[a]));
        // grad . n > 0 with n = -1 / +1 along the axis
        const bool upExt = side ? grad > 0.0 : grad < 0.0;
        const double lamU = upExt ? (a == 0 ? lwj : lnj) : lam[a];
        const double dlamU = upExt ? 0.0 : dlam[a];
        const double sK = Kf * grad;
        const double vel = sK * (-lamU);
        const double dvelP = (Kf * dgP) * (-lamU);
        const double dvelS = __dadd_rn((Kf * dgS) * (-lamU), (-dlamU) * sK);
        // mass flux (v . n) rho A; the neighbour's block is divided by its volume
        const double ra = side ? P.rhoArea[AXIS][a] : -P.rhoArea[AXIS][a];
        const double F = vel * ra;
        const double dFP = dvelP * ra;
        const double dFS = dvelS * ra;
        R[a] = __dadd_rn(R[a], F);
        D[a][0] = __dadd_rn(D[a][0], dFP);
        D[a][1] = __dadd_rn(D[a][1], dFS);
        Dj[2 * a] = dFP * -P.invVol;
        Dj[2 * a + 1] = dFS * -P.invVol;
    }
}


// What a face needs of the neighbour across it: p_w, K and the cached p_c, lambda_w, lambda_n.
struct NbrVals {
    double pw, K, pc, lw, ln;
};

// Neighbour values read from the global arrays (32-bit cell indices: N < 2^31).
struct NbrGlobal {
    const double2* x;
    const double* perm;
    const double* pc;   // intensive-quantity planes 0, 2, 4
    const double* lw;
    const double* ln;
    __device__ __forceinline__ NbrVals operator()(int q, int sj) const {
        (void)q;
        return {x[sj].x, perm[sj], pc[sj], lw[sj], ln[sj]};
    }
};
__device__ __forceinline__ NbrGlobal nbr_global(const double2* x, const double* perm, const double* iq, int64_t N) {
    return NbrGlobal{x, perm, iq, iq + 2 * N, iq + 4 * N};
}

// What the element of a cell needs of the cell itself.
struct OwnVals {
    double pw, Sw, K, pc, dpc, lam[2], dlam[2];
};

// One cell of a 3D grid: fluxes over its interior faces in intersection order (-x, +x, -y, +y,
// -z, +z), the implicit-Euler storage term (fvbaselocalresidual.hh:494-629), its boundary faces,
// division by the cell volume. Writes r_s and the Jacobian column of s; returns max |r_s|
// (NaN / Inf set *bad). `idx` is the cell's (i, j, k), `has` says which faces have a neighbour,
// `nb` holds the neighbours' split-order positions and `nbr` supplies their values.
template <typename JT, bool WITH_J, class NB>
__device__ __forceinline__ double assemble_core3(const Phys& P, const FaceGeo* __restrict__ geo, const int idx[3],
                                                 const bool has[6], const int nb[6], int s32, const OwnVals& o,
                                                 double2 so, const uint8_t* __restrict__ lens, double dt,
                                                 double2* __restrict__ rOut, JT* __restrict__ J, int& bad,
                                                 const NB& nbr) {
    const int64_t N = P.N;
    const double V = P.vol;
    const int n3[3] = {P.nx, P.ny, P.nz};
    const double pI[2] = {o.pw, o.pw + (o.pc - 0.0)};
    double R[2] = {0.0, 0.0};
    double D[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        if (!has[q]) continue;
        const int axis = q >> 1, side = q & 1;
        const int sj = nb[q];
        const FaceGeo G = geo[face_geo_index(n3, axis, idx[axis], side)];
        const NbrVals nv = nbr(q, sj);
        const double pwj = nv.pw, Kj = nv.K, pcj = nv.pc, lwj = nv.lw, lnj = nv.ln;
        double Dj[4];
        if (axis == 0)
            interior_face_tab<0>(P, G, side, o.K, pI, o.dpc, o.lam, o.dlam, pwj, Kj, pcj, lwj, lnj, R, D, Dj);
        else if (axis == 1)
            interior_face_tab<1>(P, G, side, o.K, pI, o.dpc, o.lam, o.dlam, pwj, Kj, pcj, lwj, lnj, R, D, Dj);
        else
            interior_face_tab<2>(P, G, side, o.K, pI, o.dpc, o.lam, o.dlam, pwj, Kj, pcj, lwj, lnj, R, D, Dj);
        if (WITH_J) store_block(J, N, opposite_band(band_of(axis, side)), sj, Dj);
    }
    // storage: (phi S rho - storage(x_old)) V / dt
    {
        const double Sw = o.Sw;
        const double fac = V / dt;
        const double sw0 = P.porosity * Sw * P.rho[0];
        const double sn0 = P.porosity * (1.0 - (0.0 + Sw)) * P.rho[1];
        R[0] = __dadd_rn(R[0], __dmul_rn(sw0 - so.x, fac));
        R[1] = __dadd_rn(R[1], __dmul_rn(sn0 - so.y, fac));
        D[0][1] = __dadd_rn(D[0][1], __dmul_rn(P.porosity * P.rho[0], fac));
        D[1][1] = __dadd_rn(D[1][1], __dmul_rn(-P.porosity * P.rho[1], fac));
    }
    // boundary faces (warp-uniform except at the two ends of each x-row)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        if (has[q]) continue;
        const int axis = q >> 1, side = q & 1;
        const int li = lens[s32];
        if (axis == 0)
            boundary_face<3, 0>(P, side, idx, li, o.K, pI, o.dpc, o.lam, o.dlam, R, D);
        else if (axis == 1)
            boundary_face<3, 1>(P, side, idx, li, o.K, pI, o.dpc, o.lam, o.dlam, R, D);
        else
            boundary_face<3, 2>(P, side, idx, li, o.K, pI, o.dpc, o.lam, o.dlam, R, D);
    }
    const double invV = P.invVol;
    R[0] *= invV;
    R[1] *= invV;
    rOut[s32] = make_double2(R[0], R[1]);
    if (WITH_J) {
        const double blk[4] = {D[0][0] * invV, D[0][1] * invV, D[1][0] * invV, D[1][1] * invV};
        store_block(J, N, 0, s32, blk);
    }
    if (!(fabs(R[0]) <= 1.7976931348623157e308) || !(fabs(R[1]) <= 1.7976931348623157e308)) bad = 1;
    return fmax(fabs(R[0]), fabs(R[1]));
}

// One cell of a 3D grid at split-order position s: its own intensive quantities evaluated here
// (for the S_w = 1 cells a table read, intensive_values), the neighbours' read from the global
// arrays and the cache (planes 0, 2, 4).
template <typename JT, bool WITH_J, class NB>
__device__ __forceinline__ double assemble_cell3(const Phys& P, const FaceGeo* __restrict__ geo,
                                                 const double2* __restrict__ x, const double2* __restrict__ sold,
                                                 const double* __restrict__ perm, const uint8_t* __restrict__ lens,
                                                 const double* __restrict__ iq, double dt, double2* __restrict__ rOut,
                                                 JT* __restrict__ J, int64_t s, int& bad, const NB& nbr) {
    const int s32 = (int)s;  // N < 2^31: 32-bit cell indices
    const int Nh32 = (int)P.Nh;
    const int col = s32 >= Nh32 ? 1 : 0;
    const int h = s32 - col * Nh32;
    const CellIdx ci = cell_of(P, col, h);
    const int idx[3] = {ci.i, ci.j, ci.k};
    const bool has[6] = {ci.i > 0, ci.i < P.nx - 1, ci.j > 0, ci.j < P.ny - 1, ci.k > 0, ci.k < P.nz - 1};
    const double2 xi = x[s32];
    const IqVals q = intensive_values(P, xi.y, lens[s32]);
    OwnVals o;
    o.pw = xi.x;
    o.Sw = xi.y;
    o.K = perm[s32];
    o.pc = q.pc;
    o.dpc = q.dpc;
    o.lam[0] = q.lw;
    o.lam[1] = q.ln;
    o.dlam[0] = q.dlw;
    o.dlam[1] = q.dln;
    const int base = (col ^ 1) * Nh32;
    const int nxh = P.nxh, planeh = (int)P.planeh;
    const int nb[6] = {base + h - 1 + ci.b, base + h + ci.b, base + h - nxh, base + h + nxh, base + h - planeh,
                       base + h + planeh};
    return assemble_core3<JT, WITH_J>(P, geo, idx, has, nb, s32, o, sold[s32], lens, dt, rOut, J, bad, nbr);
}

}  // namespace ewg
