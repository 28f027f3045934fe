// Device physics of the immiscible two-phase lens problem.
//
// Every per-cell quantity depends on the cell's own (p_w, S_w) only, and p_w enters linearly, so
// instead of a general 2-derivative AD type the kernels carry a value and its derivative with
// respect to S_w (struct VD) and add the trivial p_w derivatives by hand. The arithmetic follows
// the forward-mode rules of DenseAd::Evaluation (product rule, pow(x, e)' = pow(x, e)/x*e with the
// x == 0 special case, sqrt' = 0.5/sqrt) so values agree with an AD evaluation to rounding.
// Sums of products are written with explicitly rounded operations (no fused multiply-add): the
// compiler's choice of which product to fuse may differ between the kernels that inline these
// functions, and explicit rounding makes every kernel get the same bits (also the bits of an
// unfused CPU evaluation).
//
// Material laws (ewoms-material, restated from their published form):
//   EffToAbsLaw: S_e = (S - S_r) / (1 - (S_wr + S_nr)); k_rn reads 1 - S_n,e
//   RegularizedVanGenuchten: p_c = ((S_e^(-1/m) - 1)^(1/n)) / alpha on [0.01, 0.99], linear
//     extension below 0.01 with the finite-difference slope, cubic Hermite segment on (0.99, 1)
//     and a straight line beyond 1; k_rw = sqrt(S_e) (1 - (1 - S_e^(1/m))^m)^2,
//     k_rn = (1 - S_e)^(1/3) (1 - S_e^(1/m))^(2m), clamped outside (0, 1)
//   RegularizedBrooksCorey: p_c = p_e S_e^(-1/lambda) with linear extensions below 0.01 and
//     beyond 1; k_rw = S_e^(2/lambda + 3), k_rn = (1 - S_e)^2 (1 - S_e^(2/lambda + 1))
#pragma once

#include <math.h>

#include "ewg_internal.cuh"

namespace ewg {

struct VD {
    double v, d;
};

__device__ __forceinline__ VD vd_mul(VD a, VD b) {
    return {__dmul_rn(a.v, b.v), __dadd_rn(__dmul_rn(a.d, b.v), __dmul_rn(b.d, a.v))};
}
__device__ __forceinline__ VD vd_add(VD a, VD b) { return {__dadd_rn(a.v, b.v), __dadd_rn(a.d, b.d)}; }
__device__ __forceinline__ VD vd_sub(VD a, VD b) { return {__dsub_rn(a.v, b.v), __dsub_rn(a.d, b.d)}; }
__device__ __forceinline__ VD vd_scale(VD a, double s) { return {__dmul_rn(a.v, s), __dmul_rn(a.d, s)}; }
__device__ __forceinline__ VD vd_rsub(double s, VD a) { return {__dsub_rn(s, a.v), -a.d}; }  // s - a
__device__ __forceinline__ VD vd_pow(VD x, double e) {
    if (x.v == 0.0) return {0.0, 0.0};
    double px = pow(x.v, e);
    double df = px / x.v * e;
    return {px, df * x.d};
}
__device__ __forceinline__ VD vd_sqrt(VD x) {
    double s = sqrt(x.v);
    double df = 0.5 / s;
    return {s, df * x.d};
}

__device__ __forceinline__ VD vg_pcnw(const LawDev& L, VD Se) {
    VD a = vd_pow(Se, L.negInvM);
    VD b = {a.v - 1.0, a.d};
    VD c = vd_pow(b, L.invN);
    return {c.v / L.alpha, c.d / L.alpha};
}
__device__ __forceinline__ VD vg_krw(const LawDev& L, VD Se) {
    VD u = vd_pow(Se, L.invM);
    VD q = vd_pow(vd_rsub(1.0, u), L.m);
    VD r = vd_rsub(1.0, q);
    return vd_mul(vd_mul(vd_sqrt(Se), r), r);
}
__device__ __forceinline__ VD vg_krn(const LawDev& L, VD Sw) {
    VD f = vd_pow(vd_rsub(1.0, Sw), 1.0 / 3);
    VD u = vd_pow(Sw, L.invM);
    VD g = vd_pow(vd_rsub(1.0, u), L.twoM);
    return vd_mul(f, g);
}
__device__ __forceinline__ VD hermite(const LawDev& L, VD x) {
    VD t = {(x.v - L.spX0) / L.spH, x.d / L.spH};
    VD t2 = vd_mul(t, t);
    VD t3 = vd_mul(t2, t);
    VD h00 = vd_add(vd_sub(vd_scale(t3, 2.0), vd_scale(t2, 3.0)), VD{1.0, 0.0});
    VD h10 = vd_add(vd_sub(t3, vd_scale(t2, 2.0)), t);
    VD h01 = vd_add(vd_scale(t3, -2.0), vd_scale(t2, 3.0));
    VD h11 = vd_sub(t3, t2);
    VD y = vd_scale(h00, L.spY0);
    y = vd_add(y, vd_scale(h10, L.spHM0));
    y = vd_add(y, vd_scale(h01, L.spY1));
    y = vd_add(y, vd_scale(h11, L.spHM1));
    return y;
}
__device__ __forceinline__ VD reg_vg_pcnw(const LawDev& L, VD Se) {
    if (Se.v < L.pcLowSw)
        return {__dadd_rn(L.pcLow, __dmul_rn(L.pcSlopeLow, Se.v - L.pcLowSw)), L.pcSlopeLow * Se.d};
    if (Se.v > L.pcHighSw) {
        if (Se.v < 1.0) return hermite(L, Se);
        return {__dadd_rn(__dmul_rn(L.m1High, Se.v - 1.0), 0.0), L.m1High * Se.d};
    }
    return vg_pcnw(L, Se);
}
__device__ __forceinline__ VD reg_vg_krw(const LawDev& L, VD Se) {
    if (Se.v <= 0) return {0.0, 0.0};
    if (Se.v >= 1) return {1.0, 0.0};
    return vg_krw(L, Se);
}
__device__ __forceinline__ VD reg_vg_krn(const LawDev& L, VD Sw) {
    if (Sw.v <= 0) return {1.0, 0.0};
    if (Sw.v >= 1) return {0.0, 0.0};
    return vg_krn(L, Sw);
}
__device__ __forceinline__ VD reg_bc_pcnw(const LawDev& L, VD Se) {
    if (Se.v <= L.bcLowSw)
        return {__dadd_rn(L.bcPcLow, __dmul_rn(L.bcSlopeLow, Se.v - L.bcLowSw)), L.bcSlopeLow * Se.d};
    if (Se.v >= 1.0) return {__dadd_rn(L.pe, __dmul_rn(L.bcSlopeOne, Se.v - 1.0)), L.bcSlopeOne * Se.d};
    return vd_scale(vd_pow(Se, L.negInvLambda), L.pe);
}
__device__ __forceinline__ VD reg_bc_krw(const LawDev& L, VD Se) {
    if (Se.v <= 0) return {0.0, 0.0};
    if (Se.v >= 1) return {1.0, 0.0};
    return vd_pow(Se, L.krwExp);
}
__device__ __forceinline__ VD reg_bc_krn(const LawDev& L, VD Sw) {
    if (Sw.v >= 1) return {0.0, 0.0};
    if (Sw.v <= 0) return {1.0, 0.0};
    VD a = vd_pow(vd_rsub(1.0, Sw), 2.0);
    VD b = vd_rsub(1.0, vd_pow(Sw, L.krnExp));
    return vd_mul(a, b);
}

// EffToAbsLaw over the regularised law: capillary pressure p_cnw and relative permeabilities at
// absolute wetting saturation S_w, each with d/dS_w.
struct MatOut {
    VD pc, krw, krn;
};
__device__ __forceinline__ MatOut material(const LawDev& L, double Sw) {
    VD sw{Sw, 1.0};
    VD Sew = {(sw.v - L.swr) / L.den, 1.0 / L.den};
    VD Sn = vd_rsub(1.0, sw);
    VD Sen = {(Sn.v - L.snr) / L.den, Sn.d / L.den};
    VD Swn = vd_rsub(1.0, Sen);
    MatOut o;
    if (L.kind == EWG_LAW_VAN_GENUCHTEN) {
        o.pc = reg_vg_pcnw(L, Sew);
        o.krw = reg_vg_krw(L, Sew);
        o.krn = reg_vg_krn(L, Swn);
    } else {
        o.pc = reg_bc_pcnw(L, Sew);
        o.krw = reg_bc_krw(L, Sew);
        o.krn = reg_bc_krn(L, Swn);
    }
    return o;
}

// ewoms-common harmonicMean
__device__ __forceinline__ double harmonic_mean(double x, double y) {
    if (x * y <= 0) return 0.0;
    return (2 * x * y) / (y + x);
}

__device__ __forceinline__ bool in_lens(const Phys& P, const double x[3]) {
    for (int a = 0; a < P.dim; ++a)
        if (x[a] < P.lensLo[a] - P.eps || x[a] > P.lensHi[a] + P.eps) return false;
    return true;
}

}  // namespace ewg
