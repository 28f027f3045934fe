// Vertex-centred finite volumes (VcfvDiscretization with P1 finite-element gradients,
// discretizations/vcfv/) for the immiscible two-phase lens problem on the device: the AD
// linearization and a BiCGStab / block-Jacobi Newton solve.
//
// DOFs sit at the grid vertices (natural order, x fastest). Each element (an axis-aligned box)
// gives every corner a sub-control volume (SCV) and has one sub-control-volume face (SCVF) per
// edge, joining the element centre to the edge; the flux over it uses the P1 gradient of the
// phase pressures at the face's integration point (p1fegradientcalculator.hh:255-290), the
// gravity correction between the edge's two vertices, the harmonic-mean permeability of the two
// vertices and the upstream mobility (darcyfluxmodule.hh:185-324, 461-527). Boundary sub-faces
// carry the lens problem's free-flow and inlet conditions (vcfvstencil.hh:962-1012,
// darcyfluxmodule.hh:333-453, lensproblem.hh:464-533).
//
// Linearization (fvbaselinearizer.hh:401-512 with fvbaseadlocallinearizer.hh:178-297): the
// reference evaluates every element's local residual once per focus vertex and scatters
// residual_[i] += r_i, J[j][i] += dR_j/dx_i element by element. Here one thread owns one
// vertex row: it visits the (up to 2^dim) elements around its vertex in element order and, in
// each, evaluates the SCVFs that touch its vertex, the storage term of its SCV and its boundary
// sub-faces, with the derivatives with respect to each of the element's vertices; divides by the
// vertex's control volume and adds the element's contribution to its residual and to the 27 (3D)
// or 9 (2D) Jacobian blocks of its row, which it accumulates in shared memory and writes once.
// The per-face arithmetic follows the forward-mode AD rules in the reference's operation order,
// and the sums run in the reference's element order, so the outputs equal the CPU restatement's
// to rounding of the individual products (the potential gradients, whose sign picks the upstream
// vertex, are formed with explicitly rounded products and sums as on the CPU).
//
// Jacobian storage: band-major, band (dx+1) + 3 (dy+1) [+ 9 (dz+1)] for the neighbour at vertex
// offset (dx, dy, dz), 4 planes per band ([eq][pv]), each plane NV doubles.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ewg_assemble.cuh"

namespace ewg {

// Geometry of the structured element (relative to its lower corner), the same for every element.
struct VGeomDev {
    int dim, nv, ne;
    int ei[12], ej[12], axis[12];
    double nsign[12];     // the SCVF unit normal is nsign * e_axis (from ei to ej)
    double area[12];
    double G[12][8];      // axis component of the P1 gradient of vertex v at the SCVF's integration point
    double gtab[12][2];   // gravity part of the potential gradient (axis component) per phase
    double scvVol;
    double bcoef[6][8];   // boundary sub-face of (face, vertex): (ip - SCV centre)_axis / |ip - SCV centre|^2
    double bip[6][8][3];  // its integration point, local coordinates
    double barea[6][8];
};

struct VDims {
    int nvx, nvy, nvz;    // vertices per axis (nvz = 1 in 2D)
    int nex, ney, nez;    // elements per axis
    int NV;
};

}  // namespace ewg

struct ewg_vcfv {
    ewg::Phys P;            // problem constants; P.N = number of vertices (plane stride of iq)
    ewg::VDims D{};
    int nb = 9;             // Jacobian bands
    int device = 0;
    int numSMs = 148;
    cudaStream_t stream = nullptr;
    std::string err;
    ewg::VGeomDev hgeo{};
    ewg::VGeomDev* geo = nullptr;
    double2 *x0 = nullptr, *x1 = nullptr, *sold = nullptr, *r = nullptr;
    double *perm = nullptr, *totVol = nullptr, *iq = nullptr, *J = nullptr;
    double* kedge = nullptr;  // harmonic-mean permeability of each edge, plane per axis, at the lower vertex
    uint8_t* lens = nullptr;
    unsigned long long* d_errmax = nullptr;
    int* d_flags = nullptr;
    // solver vectors (2 NV doubles each) and reduction scratch
    double *s_b = nullptr, *s_x = nullptr, *s_r = nullptr, *s_r0 = nullptr, *s_v = nullptr, *s_p = nullptr,
           *s_y = nullptr, *s_z = nullptr, *s_t = nullptr, *s_dinv = nullptr, *s_red = nullptr;
    double* h_red = nullptr;  // pinned
    double* M = nullptr;      // block ILU(0) factors in the band layout (allocated at the first ILU solve)
    int precond = EWG_PRECOND_JACOBI;  // preconditioner of the current solve
    long long launches = 0;
    // the ILU(0) application (colour sweeps, relaxation) captured once per input / output / w:
    // the solve applies it to p -> y and s -> z, so two graphs serve every iteration
    struct PrecGraph {
        const double* d = nullptr;
        double* out = nullptr;
        double w = 0.0;
        int kernels = 0;
        cudaGraphExec_t exec = nullptr;
    } precGraphs[2];
    int precGraphNext = 0;
    // LocalLinearizerSplice and NumericDifferenceMethod; the reference pressure of
    // ImmiscibleModel::updateBegin (p_w of vertex 0) for the FD pressure weight, unset until then
    int localLinearizer = EWG_LOCAL_LINEARIZER_AD;
    int fdMethod = 1;
    double refPressure = -1.0;
};

namespace ewg {

static ewg_status vfail(ewg_vcfv* c, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EWG_OK;
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return EWG_ERR_CUDA;
}

// ---- geometry (host), the operations of the CPU restatement --------------------------------

static void vcross(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static void vquad_normal(const double p0[3], const double p1[3], const double p2[3], const double p3[3], double n[3]) {
    double a[3], b[3];
    for (int d = 0; d < 3; ++d) { a[d] = p2[d] - p0[d]; b[d] = p3[d] - p1[d]; }
    vcross(a, b, n);
    for (int d = 0; d < 3; ++d) n[d] *= 0.5;
}
static double vnorm(const double n[3], int dim) {
    double s = 0.0;
    for (int d = 0; d < dim; ++d) s += n[d] * n[d];
    return std::sqrt(s);
}

static VGeomDev build_vgeom(const Phys& P) {
    VGeomDev g;
    memset(&g, 0, sizeof(g));
    const int dim = P.dim;
    double h[3];
    for (int d = 0; d < 3; ++d) h[d] = d < dim ? P.h[d] : 1.0;
    g.dim = dim;
    g.nv = 1 << dim;
    g.ne = dim == 2 ? 4 : 12;
    const int nf = 2 * dim;
    int vb[8][3];
    for (int v = 0; v < g.nv; ++v)
        for (int d = 0; d < 3; ++d) vb[v][d] = d < dim ? (v >> d) & 1 : 0;
    auto glob = [&](const double l[3], double o[3]) { for (int d = 0; d < 3; ++d) o[d] = d < dim ? l[d] * h[d] : 0.0; };
    double elemL[3] = {0.5, 0.5, dim == 3 ? 0.5 : 0.0}, elemG[3];
    glob(elemL, elemG);
    double faceL[6][3], faceG[6][3];
    int faxis[6], fside[6];
    for (int f = 0; f < nf; ++f) {
        int a = f >> 1, sd = f & 1;
        faxis[f] = a; fside[f] = sd;
        for (int d = 0; d < 3; ++d) faceL[f][d] = d < dim ? 0.5 : 0.0;
        faceL[f][a] = sd;
        glob(faceL[f], faceG[f]);
    }
    static const int e2[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};
    static const int e3[12][2] = {{0, 4}, {1, 5}, {2, 6}, {3, 7}, {0, 2}, {1, 3},
                                  {0, 1}, {2, 3}, {4, 6}, {5, 7}, {4, 5}, {6, 7}};
    static const unsigned edgeToFaceHex[2][12] = {{0, 2, 3, 1, 4, 1, 2, 4, 0, 5, 5, 3},
                                                  {2, 1, 0, 3, 0, 4, 4, 3, 5, 1, 2, 5}};
    double edgeL[12][3], edgeG[12][3];
    double ipL[12][3];
    for (int k = 0; k < g.ne; ++k) {
        int a = dim == 2 ? e2[k][0] : e3[k][0], b = dim == 2 ? e2[k][1] : e3[k][1];
        for (int d = 0; d < 3; ++d) edgeL[k][d] = d < dim ? 0.5 * (vb[a][d] + vb[b][d]) : 0.0;
        glob(edgeL[k], edgeG[k]);
        int i = a, j = b;
        if (g.ne == 4 && (i == 2 || j == 2)) std::swap(i, j);
        g.ei[k] = i; g.ej[k] = j;
        double n[3] = {0, 0, 0};
        if (dim == 2) {
            for (int d = 0; d < 3; ++d) ipL[k][d] = (edgeL[k][d] + elemL[d]) * 0.5;
            double diff[3];
            for (int d = 0; d < 2; ++d) diff[d] = elemG[d] - edgeG[k][d];
            n[0] = diff[1]; n[1] = -diff[0];
            double xi[3], xj[3], li[3], lj[3];
            for (int d = 0; d < 3; ++d) { li[d] = vb[i][d]; lj[d] = vb[j][d]; }
            glob(li, xi); glob(lj, xj);
            double dot = 0.0;
            for (int d = 0; d < 2; ++d) dot += n[d] * (xj[d] - xi[d]);
            if (dot < 0) for (int d = 0; d < 2; ++d) n[d] *= -1;
        } else {
            unsigned lf = edgeToFaceHex[0][k], rf = edgeToFaceHex[1][k];
            for (int d = 0; d < 3; ++d) ipL[k][d] = (((edgeL[k][d] + elemL[d]) + faceL[lf][d]) + faceL[rf][d]) * 0.25;
            vquad_normal(edgeG[k], faceG[rf], elemG, faceG[lf], n);
        }
        g.area[k] = vnorm(n, dim);
        int ax = 0;
        for (int d = 0; d < dim; ++d) if (vb[i][d] != vb[j][d]) ax = d;
        g.axis[k] = ax;
        g.nsign[k] = n[ax] / g.area[k];
        // P1 (Q1) shape-function gradients at the integration point, axis component
        for (int v = 0; v < g.nv; ++v) {
            double q = vb[v][ax] ? 1.0 : -1.0;
            for (int e = 0; e < dim; ++e)
                if (e != ax) q *= vb[v][e] ? ipL[k][e] : 1.0 - ipL[k][e];
            g.G[k][v] = (1.0 / h[ax]) * q;
        }
        // gravity correction between the vertices, at the integration point
        double posIn[3], posEx[3], posF[3], distIn[3], distEx[3], distTot[3];
        for (int d = 0; d < 3; ++d) {
            posIn[d] = vb[i][d] * h[d];
            posEx[d] = vb[j][d] * h[d];
            posF[d] = ipL[k][d] * h[d];
        }
        for (int d = 0; d < 3; ++d) { distIn[d] = posIn[d] - posF[d]; distEx[d] = posEx[d] - posF[d]; distTot[d] = posEx[d] - posIn[d]; }
        double absDistTotSq = 0.0;
        for (int d = 0; d < dim; ++d) absDistTotSq += distTot[d] * distTot[d];
        double gIn = 0.0, gEx = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double gd = d == 1 ? -P.g : 0.0;
            gIn += gd * distIn[d];
            gEx += gd * distEx[d];
        }
        for (int ph = 0; ph < 2; ++ph) {
            const double pStatIn = -(P.rho[ph] * gIn);
            const double pStatEx = -(P.rho[ph] * gEx);
            const double qq = (pStatEx - pStatIn) / absDistTotSq;
            g.gtab[k][ph] = distTot[ax] * qq;
        }
    }
    double vol = 1.0;
    for (int d = 0; d < dim; ++d) vol *= h[d];
    g.scvVol = vol / g.nv;
    static const int leftEdgeHex[6][8] = {{0, -1, 4, -1, 8, -1, 2, -1}, {-1, 5, -1, 3, -1, 1, -1, 9},
                                          {6, 1, -1, -1, 0, 10, -1, -1}, {-1, -1, 2, 7, -1, -1, 11, 3},
                                          {4, 6, 7, 5, -1, -1, -1, -1}, {-1, -1, -1, -1, 10, 9, 8, 11}};
    static const int rightEdgeHex[6][8] = {{4, -1, 2, -1, 0, -1, 8, -1}, {-1, 1, -1, 5, -1, 9, -1, 3},
                                           {0, 6, -1, -1, 10, 1, -1, -1}, {-1, -1, 7, 3, -1, -1, 2, 11},
                                           {6, 5, 4, 7, -1, -1, -1, -1}, {-1, -1, -1, -1, 8, 10, 11, 9}};
    for (int f = 0; f < nf; ++f)
        for (int v = 0; v < g.nv; ++v) {
            if (vb[v][faxis[f]] != fside[f]) continue;
            double vl[3] = {(double)vb[v][0], (double)vb[v][1], (double)vb[v][2]};
            double ip[3];
            if (dim == 2) {
                for (int d = 0; d < 3; ++d) ip[d] = (vl[d] + faceL[f][d]) * 0.5;
                g.barea[f][v] = 0.5 * h[1 - faxis[f]];
            } else {
                int le = leftEdgeHex[f][v], re = rightEdgeHex[f][v];
                for (int d = 0; d < 3; ++d) ip[d] = (((vl[d] + faceL[f][d]) + edgeL[le][d]) + edgeL[re][d]) * 0.25;
                double vg[3], n[3];
                glob(vl, vg);
                vquad_normal(vg, edgeG[re], faceG[f], edgeG[le], n);
                g.barea[f][v] = vnorm(n, 3);
            }
            for (int d = 0; d < 3; ++d) g.bip[f][v][d] = ip[d];
            // two-point boundary gradient from the SCV centre to the integration point
            double ipG[3], scvC[3];
            for (int d = 0; d < 3; ++d) {
                ipG[d] = ip[d] * h[d];
                const double cl = d < dim ? (vb[v][d] + elemL[d]) * 0.5 : 0.0;
                scvC[d] = cl * h[d];
            }
            double distSq = 0.0;
            for (int d = 0; d < dim; ++d) { double t = ipG[d] - scvC[d]; distSq += t * t; }
            const double t = ipG[faxis[f]] - scvC[faxis[f]];
            g.bcoef[f][v] = t / distSq;
        }
    return g;
}

// ---- device ---------------------------------------------------------------------------------

constexpr int kVBlock = 64;       // vertex rows per block of the assembly kernel
constexpr int kVApi = 256;

__global__ void kv_intensive(const __grid_constant__ Phys P, const double2* __restrict__ x,
                             const uint8_t* __restrict__ lens, double* __restrict__ iq) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x)
        intensive_cell(P, x, lens, iq, s);
}

// storage per unit volume of a state (ImmiscibleLocalResidual::computeStorage)
__global__ void kv_storage(const __grid_constant__ Phys P, const double2* __restrict__ x, double2* __restrict__ out) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < P.N; s += (int64_t)gridDim.x * blockDim.x) {
        const double Sw = x[s].y;
        out[s] = make_double2(P.porosity * Sw * P.rho[0], P.porosity * (1.0 - (0.0 + Sw)) * P.rho[1]);
    }
}

// LensProblem::initial at the vertex positions
__global__ void kv_initial(const __grid_constant__ Phys P, VDims D, double2* __restrict__ x) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < D.NV; v += gridDim.x * blockDim.x) {
        const int j = (v / D.nvx) % D.nvy;
        const double y = j * P.h[1];
        const double depth = P.L[1] - y;
        x[v] = make_double2(P.pRef - P.rho[0] * (-P.g) * depth, 1.0);
    }
}

// dofTotalVolume: the SCV volumes of the adjacent elements, summed in element order
__global__ void kv_total_volume(VDims D, int dim, double scvVol, double* __restrict__ out) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < D.NV; v += gridDim.x * blockDim.x) {
        const int i = v % D.nvx, j = (v / D.nvx) % D.nvy, k = v / (D.nvx * D.nvy);
        double s = 0.0;
        for (int oz = (dim == 3 ? -1 : 0); oz <= 0; ++oz)
            for (int oy = -1; oy <= 0; ++oy)
                for (int ox = -1; ox <= 0; ++ox) {
                    const int ex = i + ox, ey = j + oy, ez = k + oz;
                    if (ex < 0 || ey < 0 || ez < 0 || ex >= D.nex || ey >= D.ney || ez >= D.nez) continue;
                    s += scvVol * 1.0;
                }
        out[v] = s;
    }
}

// the face permeability of every edge, harmonic mean of its two vertices (symmetric in its
// arguments, so either end gets the same value), stored at the edge's lower vertex per axis
__global__ void kv_edge_perm(VDims D, int dim, const double* __restrict__ perm, double* __restrict__ kedge) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < D.NV; v += gridDim.x * blockDim.x) {
        const int i = v % D.nvx, j = (v / D.nvx) % D.nvy, k = v / (D.nvx * D.nvy);
        const int id[3] = {i, j, k}, n[3] = {D.nvx, D.nvy, D.nvz}, st[3] = {1, D.nvx, D.nvx * D.nvy};
        for (int ax = 0; ax < 3; ++ax)
            kedge[(int64_t)ax * D.NV + v] = ax < dim && id[ax] + 1 < n[ax] ? harmonic_mean(perm[v], perm[v + st[ax]]) : 0.0;
    }
}

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

// SCVF endpoints (interior i, exterior j) of the structured element, as build_vgeom orders them
__device__ constexpr int kEdge2[4][2] = {{2, 0}, {1, 3}, {0, 1}, {3, 2}};
__device__ constexpr int kEdge3[12][2] = {{0, 4}, {1, 5}, {2, 6}, {3, 7}, {0, 2}, {1, 3},
                                          {0, 1}, {2, 3}, {4, 6}, {5, 7}, {4, 5}, {6, 7}};

// Element contribution to the row of local vertex A (compile time) of the element at offset
// (ox, oy, oz) from the thread's vertex, added to r and to the shared-memory block accumulators:
// the SCVFs touching A (edge order, resolved at compile time), the storage of A's SCV and A's
// boundary sub-faces, scaled by 1 / A's control volume. The potential gradient, whose sign picks the
// upstream vertex, is summed with explicitly rounded operations in the reference's order; the flux
// factor K_f (-lambda) n rho |A| is formed once per face and phase, so every derivative is one or
// two products (the same values to a few ulps).
template <int DIM, int A>
__device__ __forceinline__ void vcfv_element(const Phys& P, const VDims& D, const VGeomDev* __restrict__ geo,
                                             const double2* __restrict__ x, const double2* __restrict__ sold,
                                             const double* __restrict__ perm, const uint8_t* __restrict__ lens,
                                             const double* __restrict__ iq, const double* __restrict__ kedge,
                                             double cst, double V, int v,
                                             const int eidx[3], double r[2], double* acc, int& bad) {
    constexpr int NV = 1 << DIM;
    constexpr int NE = DIM == 3 ? 12 : 4;
    const int64_t NVt = D.NV;
    const int sy = D.nvx, sz = D.nvx * D.nvy;
    auto gidx = [&](int w) {
        const int dx = (w & 1) - (A & 1), dy = ((w >> 1) & 1) - ((A >> 1) & 1);
        const int dz = DIM == 3 ? ((w >> 2) & 1) - ((A >> 2) & 1) : 0;
        return v + dx + sy * dy + sz * dz;
    };
    double pw[NV], pn[NV], dpc[NV];
#pragma unroll
    for (int w = 0; w < NV; ++w) {
        const int g = gidx(w);
        pw[w] = x[g].x;
        pn[w] = pw[w] + (iq[g] - 0.0);
        dpc[w] = iq[NVt + g];
    }
    double Rv[2] = {0.0, 0.0};
    double Rd[NV][2][2];
#pragma unroll
    for (int w = 0; w < NV; ++w) Rd[w][0][0] = Rd[w][0][1] = Rd[w][1][0] = Rd[w][1][1] = 0.0;
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        const int i = DIM == 3 ? kEdge3[k][0] : kEdge2[k][0];
        const int j = DIM == 3 ? kEdge3[k][1] : kEdge2[k][1];
        if (i != A && j != A) continue;
        const bool plus = i == A;
        const double ns = geo->nsign[k];
        const double area = geo->area[k];
        const int gi = gidx(i), gj = gidx(j);
        const int ax = (i ^ j) == 1 ? 0 : ((i ^ j) == 2 ? 1 : 2);
        const double Kf = kedge[ax * NVt + (gi < gj ? gi : gj)];
        double G[NV];
#pragma unroll
        for (int w = 0; w < NV; ++w) G[w] = geo->G[k][w];
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            double g = 0.0;
#pragma unroll
            for (int w = 0; w < NV; ++w) g = dadd(g, dmul(a == 0 ? pw[w] : pn[w], G[w]));
            g = dadd(g, geo->gtab[k][a]);
            const bool upJ = dmul(g, ns) > 0.0;
            const int gu = upJ ? gj : gi;
            const double lam = iq[(a == 0 ? 2 : 4) * NVt + gu];
            const double dlam = iq[(a == 0 ? 3 : 5) * NVt + gu];
            const double nra = ns * P.rho[a] * area;        // n rho |A|
            double Cf = Kf * (-lam) * nra;                  // dF / dg
            double Dl = (-dlam) * (Kf * g) * nra;           // dF / dS of the upstream vertex via lambda
            if (!plus) { Cf = -Cf; Dl = -Dl; }
            Rv[a] += g * Cf;
#pragma unroll
            for (int w = 0; w < NV; ++w) {
                const double gc = G[w] * Cf;
                Rd[w][a][0] += gc;
                if (a == 1) Rd[w][1][1] += dpc[w] * gc;
            }
            if (upJ) Rd[j][a][1] += Dl;
            else Rd[i][a][1] += Dl;
        }
    }
    // storage of the SCV of A: (storage - storage_old) * V_scv / dt
    {
        const double Sw = x[v].y;
        const double2 so = sold[v];
        const double c = cst;
        const double stw = P.porosity * Sw * P.rho[0];
        const double stn = P.porosity * (1.0 - (0.0 + Sw)) * P.rho[1];
        Rv[0] += (stw - so.x) * c;
        Rv[1] += (stn - so.y) * c;
        Rd[A][0][1] += P.porosity * P.rho[0] * c;
        Rd[A][1][1] += -P.porosity * P.rho[1] * c;
    }
    // boundary sub-faces of A in this element (intersection order)
#pragma unroll
    for (int f = 0; f < 2 * DIM; ++f) {
        const int ax = f >> 1, sd = f & 1;
        if (((A >> ax) & 1) != sd) continue;
        const int nAx = ax == 0 ? D.nex : (ax == 1 ? D.ney : D.nez);
        if (sd == 0 ? eidx[ax] != 0 : eidx[ax] != nAx - 1) continue;
        double pos[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) pos[d] = d < DIM ? (eidx[d] + geo->bip[f][A][d]) * P.h[d] : 0.0;
        const double barea = geo->barea[f][A] * 1.0;
        const bool left = pos[0] < 0.0 + P.eps, right = pos[0] > P.L[0] - P.eps;
        if (left || right) {
            const double depth = P.L[1] - pos[1];
            const double pwB = left ? P.pRef - P.leftScale * P.rho[0] * (-P.g) * depth
                                    : P.pRef - P.rho[0] * (-P.g) * depth;
            const double pB[2] = {pwB, pwB + P.bndPc[in_lens(P, pos) ? 1 : 0] - 0.0};
            const double coef = geo->bcoef[f][A];
            const double ns = sd ? 1.0 : -1.0;
            const double K = perm[v];
            const int li = lens[v];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const double pI = a == 0 ? pw[A] : pn[A];
                const double g = dmul(pB[a] - pI, coef);
                const bool upB = dmul(g, ns) > 0.0;
                const double lam = upB ? P.bndLam[li][a] : iq[(a == 0 ? 2 : 4) * NVt + v];
                const double dlam = upB ? 0.0 : iq[(a == 0 ? 3 : 5) * NVt + v];
                const double nra = ns * P.rho[a] * barea;
                const double Cf = K * (-lam) * nra;          // d rate / d g
                Rv[a] += g * Cf;
                // dg/dp = -coef, dg/dS = -dpc coef (non-wetting phase)
                Rd[A][a][0] += -coef * Cf;
                Rd[A][a][1] += (a == 1 ? -dpc[A] * coef * Cf : 0.0) + (-dlam) * (K * g) * nra;
            }
            continue;
        }
        const bool upper = pos[1] > P.L[1] - P.eps;
        bool inlet = upper && pos[0] > P.inletXlo && pos[0] < P.inletXhi;
        if (DIM == 3) inlet = inlet && pos[2] > P.inletZlo && pos[2] < P.inletZhi;
        if (inlet) Rv[1] += P.inletRate * barea;
    }
    // volumetric residual, then the scatter into the row
    const double invV = 1.0 / V;
    r[0] += Rv[0] * invV;
    r[1] += Rv[1] * invV;
#pragma unroll
    for (int w = 0; w < NV; ++w) {
        const int dx = (w & 1) - (A & 1), dy = ((w >> 1) & 1) - ((A >> 1) & 1);
        const int dz = DIM == 3 ? ((w >> 2) & 1) - ((A >> 2) & 1) : 0;
        const int band = (dx + 1) + 3 * (dy + 1) + (DIM == 3 ? 9 * (dz + 1) : 0);
        // the dz = +1 plane reuses the dz = -1 plane's slots (flushed after the lower elements)
        const int slot = DIM == 3 && band >= 18 ? band - 18 : band;
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[(slot * 4 + e) * kVBlock] += Rd[w][e >> 1][e & 1] * invV;
    }
    if (!isfinite(Rv[0]) || !isfinite(Rv[1])) bad = 1;
}

// ---- finite-difference local linearizer (lens_immiscible_vcfv_fd) -------------------------------
//
// FvBaseFdLocalLinearizer (fvbasefdlocallinearizer.hh:221-237, 393-453) on the vertex-centred
// stencil: the element's local residual entry of vertex A at the primary variables and, per
// element vertex w and primary variable, at w's variable deflected by eps = BaseEpsilon /
// primaryVarWeight (weight 10 / p_ref for the pressure, 1 for the saturation); only w's intensive
// quantities are re-evaluated, the storage of the previous time level is read from the cache.
// Values only: the same face arithmetic as the AD kernel.

template <int DIM>
struct VcfvElemState {
    double pw[1 << DIM], pn[1 << DIM], lw[1 << DIM], ln[1 << DIM];
    double SwA;
};
// p_c, lambda_w, lambda_n at the primary variables (a pressure deflection keeps them)
template <int DIM>
struct VcfvElemIq {
    double pc[1 << DIM];
};

// local residual entry of vertex A (compile time) in the element, scaled by 1 / control volume
template <int DIM, int A>
__device__ __forceinline__ void vcfv_local_value(const Phys& P, const VDims& D, const VGeomDev* __restrict__ geo,
                                                 const double* __restrict__ kedge, double cst, double invV, int v,
                                                 const int eidx[3], const VcfvElemState<DIM>& st, double2 so, double KA,
                                                 int liA, double R[2]) {
    constexpr int NV = 1 << DIM;
    constexpr int NE = DIM == 3 ? 12 : 4;
    const int64_t NVt = D.NV;
    const int sy = D.nvx, sz = D.nvx * D.nvy;
    auto gidx = [&](int w) {
        const int dx = (w & 1) - (A & 1), dy = ((w >> 1) & 1) - ((A >> 1) & 1);
        const int dz = DIM == 3 ? ((w >> 2) & 1) - ((A >> 2) & 1) : 0;
        return v + dx + sy * dy + sz * dz;
    };
    double Rv[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        const int i = DIM == 3 ? kEdge3[k][0] : kEdge2[k][0];
        const int j = DIM == 3 ? kEdge3[k][1] : kEdge2[k][1];
        if (i != A && j != A) continue;
        const double ns = geo->nsign[k];
        const double area = geo->area[k];
        const int gi = gidx(i), gj = gidx(j);
        const int ax = (i ^ j) == 1 ? 0 : ((i ^ j) == 2 ? 1 : 2);
        const double Kf = kedge[ax * NVt + (gi < gj ? gi : gj)];
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            double g = 0.0;
#pragma unroll
            for (int w = 0; w < NV; ++w) g = dadd(g, dmul(a == 0 ? st.pw[w] : st.pn[w], geo->G[k][w]));
            g = dadd(g, geo->gtab[k][a]);
            const bool upJ = dmul(g, ns) > 0.0;
            const double lam = a == 0 ? (upJ ? st.lw[j] : st.lw[i]) : (upJ ? st.ln[j] : st.ln[i]);
            const double nra = ns * P.rho[a] * area;
            const double F = g * (Kf * (-lam) * nra);
            Rv[a] += i == A ? F : -F;
        }
    }
    {
        const double stw = P.porosity * st.SwA * P.rho[0];
        const double stn = P.porosity * (1.0 - (0.0 + st.SwA)) * P.rho[1];
        Rv[0] += (stw - so.x) * cst;
        Rv[1] += (stn - so.y) * cst;
    }
#pragma unroll
    for (int f = 0; f < 2 * DIM; ++f) {
        const int ax = f >> 1, sd = f & 1;
        if (((A >> ax) & 1) != sd) continue;
        const int nAx = ax == 0 ? D.nex : (ax == 1 ? D.ney : D.nez);
        if (sd == 0 ? eidx[ax] != 0 : eidx[ax] != nAx - 1) continue;
        double pos[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) pos[d] = d < DIM ? (eidx[d] + geo->bip[f][A][d]) * P.h[d] : 0.0;
        const double barea = geo->barea[f][A] * 1.0;
        const bool left = pos[0] < 0.0 + P.eps, right = pos[0] > P.L[0] - P.eps;
        if (left || right) {
            const double depth = P.L[1] - pos[1];
            const double pwB = left ? P.pRef - P.leftScale * P.rho[0] * (-P.g) * depth
                                    : P.pRef - P.rho[0] * (-P.g) * depth;
            const double pB[2] = {pwB, pwB + P.bndPc[in_lens(P, pos) ? 1 : 0] - 0.0};
            const double coef = geo->bcoef[f][A];
            const double ns = sd ? 1.0 : -1.0;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const double g = dmul(pB[a] - (a == 0 ? st.pw[A] : st.pn[A]), coef);
                const bool upB = dmul(g, ns) > 0.0;
                const double lam = upB ? P.bndLam[liA][a] : (a == 0 ? st.lw[A] : st.ln[A]);
                Rv[a] += g * (KA * (-lam) * (ns * P.rho[a] * barea));
            }
            continue;
        }
        const bool upper = pos[1] > P.L[1] - P.eps;
        bool inlet = upper && pos[0] > P.inletXlo && pos[0] < P.inletXhi;
        if (DIM == 3) inlet = inlet && pos[2] > P.inletZlo && pos[2] < P.inletZhi;
        if (inlet) Rv[1] += P.inletRate * barea;
    }
    R[0] = Rv[0] * invV;
    R[1] = Rv[1] * invV;
}

template <int DIM, int A>
__device__ __forceinline__ void vcfv_element_fd(const Phys& P, const VDims& D, const VGeomDev* __restrict__ geo,
                                                const double2* __restrict__ x, const double2* __restrict__ sold,
                                                const double* __restrict__ perm, const uint8_t* __restrict__ lens,
                                                const double* __restrict__ iq, const double* __restrict__ kedge,
                                                double cst, double V, int v, const int eidx[3], double refPressure,
                                                int method, double r[2], double* acc, int& bad) {
    constexpr int NV = 1 << DIM;
    const int64_t NVt = D.NV;
    const int sy = D.nvx, sz = D.nvx * D.nvy;
    auto gidx = [&](int w) {
        const int dx = (w & 1) - (A & 1), dy = ((w >> 1) & 1) - ((A >> 1) & 1);
        const int dz = DIM == 3 ? ((w >> 2) & 1) - ((A >> 2) & 1) : 0;
        return v + dx + sy * dy + sz * dz;
    };
    VcfvElemState<DIM> base;
    VcfvElemIq<DIM> biq;
    double Sw[NV];
#pragma unroll
    for (int w = 0; w < NV; ++w) {
        const int g = gidx(w);
        const double2 xw = x[g];
        base.pw[w] = xw.x;
        base.pn[w] = xw.x + (iq[g] - 0.0);
        base.lw[w] = iq[2 * NVt + g];
        base.ln[w] = iq[4 * NVt + g];
        biq.pc[w] = iq[g];
        Sw[w] = xw.y;
    }
    base.SwA = Sw[A];
    const double2 so = sold[v];
    const double KA = perm[v];
    const int liA = lens[v];
    const double invV = 1.0 / V;
    double R0[2];
    vcfv_local_value<DIM, A>(P, D, geo, kedge, cst, invV, v, eidx, base, so, KA, liA, R0);
    r[0] += R0[0];
    r[1] += R0[1];
    if (!isfinite(R0[0]) || !isfinite(R0[1])) bad = 1;
    const double baseEps = fmax(0.9123e-10, 2.220446049250313e-16 * 1.23e3);
#pragma unroll
    for (int w = 0; w < NV; ++w) {
        const int dx = (w & 1) - (A & 1), dy = ((w >> 1) & 1) - ((A >> 1) & 1);
        const int dz = DIM == 3 ? ((w >> 2) & 1) - ((A >> 2) & 1) : 0;
        const int band = (dx + 1) + 3 * (dy + 1) + (DIM == 3 ? 9 * (dz + 1) : 0);
        const int slot = DIM == 3 && band >= 18 ? band - 18 : band;
        const int lw_ = lens[gidx(w)];
#pragma unroll 1
        for (int pv = 0; pv < 2; ++pv) {
            const double pvWeight = pv == 0 ? 10 / refPressure : 1.0;
            const double eps = baseEps / pvWeight;
            double pri[2] = {base.pw[w], Sw[w]};
            double delta = 0.0;
            double deriv[2];
            // w's state at deflected primary variables
            auto deflected = [&](double R[2]) {
                VcfvElemState<DIM> st = base;
                st.pw[w] = pri[0];
                if (pv == 0) {
                    // the intensive quantities depend on S_w only: those of the primary variables
                    st.pn[w] = pri[0] + (biq.pc[w] - 0.0);
                } else {
                    const IqVals o = intensive_values(P, pri[1], lw_);
                    st.pn[w] = pri[0] + (o.pc - 0.0);
                    st.lw[w] = o.lw;
                    st.ln[w] = o.ln;
                }
                if (w == A) st.SwA = pri[1];
                vcfv_local_value<DIM, A>(P, D, geo, kedge, cst, invV, v, eidx, st, so, KA, liA, R);
            };
            double Rp[2];
            if (method >= 0) {
                pri[pv] += eps;
                delta += eps;
                deflected(Rp);
                deriv[0] = Rp[0]; deriv[1] = Rp[1];
            } else {
                deriv[0] = R0[0]; deriv[1] = R0[1];
            }
            if (method <= 0) {
                pri[pv] -= delta + eps;
                delta += eps;
                deflected(Rp);
                deriv[0] -= Rp[0]; deriv[1] -= Rp[1];
            } else {
                deriv[0] -= R0[0]; deriv[1] -= R0[1];
            }
            acc[(slot * 4 + pv) * kVBlock] += deriv[0] / delta;
            acc[(slot * 4 + 2 + pv) * kVBlock] += deriv[1] / delta;
        }
    }
}

// Non-negative doubles compare like their bit patterns as unsigned integers.
__device__ __forceinline__ void vblock_max(double v, unsigned long long* out) {
    __shared__ double sm[kVBlock / 32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sm[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int q = 0; q < kVBlock / 32; ++q) m = fmax(m, sm[q]);
        atomicMax(out, (unsigned long long)__double_as_longlong(m));
    }
}

// Accumulator slots per thread: 3D rows have 27 blocks, but the 4 elements below the vertex (the
// first in element order) are the only ones that reach the dz = -1 plane and the 4 above the only
// ones that reach dz = +1, so after the lower four the dz = -1 blocks are complete, written out,
// and their slots reused: 18 blocks live at a time.
template <int DIM>
__host__ __device__ constexpr int vcfv_slots() { return DIM == 3 ? 18 : 9; }

// resident blocks per SM: the 3D AD form at four (230 registers, no spills) measured 5.73 ms per
// linearization at 256x256x128 elements against 6.21 ms at six (168 registers with spills)
template <int DIM, bool FD>
__global__ void __launch_bounds__(kVBlock, FD ? 2 : 4) kv_assemble(const __grid_constant__ Phys P, VDims D,
                                                       const VGeomDev* __restrict__ geo,
                                                       const double2* __restrict__ x, const double2* __restrict__ sold,
                                                       const double* __restrict__ perm, const uint8_t* __restrict__ lens,
                                                       const double* __restrict__ iq, const double* __restrict__ kedge,
                                                       const double* __restrict__ totVol,
                                                       double dt, double refPressure, int method,
                                                       double2* __restrict__ rOut, double* __restrict__ J,
                                                       unsigned long long* errmax, int* flags) {
    constexpr int NS = vcfv_slots<DIM>();
    extern __shared__ double vacc[];
    double* acc = vacc + threadIdx.x;
    for (int q = 0; q < NS * 4; ++q) acc[q * kVBlock] = 0.0;
    const int v = blockIdx.x * kVBlock + threadIdx.x;
    double err = 0.0;
    int bad = 0;
    if (v < D.NV) {
        const int i = v % D.nvx, j = (v / D.nvx) % D.nvy, k = v / (D.nvx * D.nvy);
        const double V = totVol[v];
        const double cst = geo->scvVol * 1.0 / dt;  // V_scv / dt of the storage term
        double r[2] = {0.0, 0.0};
        // elements around the vertex in element order; the vertex is local vertex A = ~offset bits
#define EWG_VCFV_ELEM(EO)                                                                                   \
        {                                                                                                   \
            constexpr int A = (~(EO)) & ((1 << DIM) - 1);                                                   \
            const int eidx[3] = {i - (((EO) >> 0) & 1 ? 0 : 1), j - (((EO) >> 1) & 1 ? 0 : 1),              \
                                 DIM == 3 ? k - (((EO) >> 2) & 1 ? 0 : 1) : 0};                             \
            if (eidx[0] >= 0 && eidx[1] >= 0 && eidx[2] >= 0 && eidx[0] < D.nex && eidx[1] < D.ney &&       \
                eidx[2] < D.nez)                                                                            \
            {                                                                                               \
                if (FD)                                                                                     \
                    vcfv_element_fd<DIM, A>(P, D, geo, x, sold, perm, lens, iq, kedge, cst, V, v, eidx,     \
                                            refPressure, method, r, acc, bad);                              \
                else                                                                                        \
                    vcfv_element<DIM, A>(P, D, geo, x, sold, perm, lens, iq, kedge, cst, V, v, eidx, r, acc, bad); \
            }                                                                                               \
        }
        EWG_VCFV_ELEM(0) EWG_VCFV_ELEM(1) EWG_VCFV_ELEM(2) EWG_VCFV_ELEM(3)
        if (DIM == 3) {
            // the dz = -1 blocks (bands 0..8) are complete: write them and free their slots
#pragma unroll 1
            for (int q = 0; q < 36; ++q) {
                J[(int64_t)q * D.NV + v] = acc[q * kVBlock];
                acc[q * kVBlock] = 0.0;
            }
            EWG_VCFV_ELEM(4) EWG_VCFV_ELEM(5) EWG_VCFV_ELEM(6) EWG_VCFV_ELEM(7)
        }
#undef EWG_VCFV_ELEM
        rOut[v] = make_double2(r[0], r[1]);
        if (DIM == 3) {
            for (int q = 36; q < 72; ++q) J[(int64_t)q * D.NV + v] = acc[q * kVBlock];         // dz = 0
            for (int q = 0; q < 36; ++q) J[(int64_t)(q + 72) * D.NV + v] = acc[q * kVBlock];  // dz = +1
        } else {
            for (int q = 0; q < 36; ++q) J[(int64_t)q * D.NV + v] = acc[q * kVBlock];
        }
        err = fmax(fabs(r[0]), fabs(r[1]));
        if (!(err <= 1.7976931348623157e308)) bad = 1;
    }
    if (bad) atomicOr(flags, 1);
    vblock_max(bad ? 0.0 : err, errmax);
}

// band storage -> BCRS blocks (row-major [eq][pv]) in the natural pattern
__global__ void kv_to_bcrs(VDims D, int dim, const double* __restrict__ J, const int32_t* __restrict__ rowPtr,
                           const int32_t* __restrict__ colIdx, double* __restrict__ out) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < D.NV; v += gridDim.x * blockDim.x) {
        const int i = v % D.nvx, j = (v / D.nvx) % D.nvy, k = v / (D.nvx * D.nvy);
        for (int q = rowPtr[v]; q < rowPtr[v + 1]; ++q) {
            const int c = colIdx[q];
            const int ci = c % D.nvx, cj = (c / D.nvx) % D.nvy, ck = c / (D.nvx * D.nvy);
            const int band = (ci - i + 1) + 3 * (cj - j + 1) + (dim == 3 ? 9 * (ck - k + 1) : 0);
            for (int e = 0; e < 4; ++e) out[4 * (int64_t)q + e] = J[((int64_t)band * 4 + e) * D.NV + v];
        }
    }
}

// ---- BiCGStab with block Jacobi on the band matrix ----------------------------------------------

// y = A x (2-vectors per vertex)
template <int DIM>
__global__ void kv_spmv(VDims D, const double* __restrict__ J, const double* __restrict__ x, double* __restrict__ y) {
    constexpr int NB = DIM == 3 ? 27 : 9;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < D.NV; v += gridDim.x * blockDim.x) {
        const int i = v % D.nvx, j = (v / D.nvx) % D.nvy, k = v / (D.nvx * D.nvy);
        double a0 = 0.0, a1 = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int dx = b % 3 - 1, dy = (b / 3) % 3 - 1, dz = DIM == 3 ? b / 9 - 1 : 0;
            const int ii = i + dx, jj = j + dy, kk = k + dz;
            if (ii < 0 || jj < 0 || kk < 0 || ii >= D.nvx || jj >= D.nvy || kk >= D.nvz) continue;
            const int c = v + dx + D.nvx * (dy + D.nvy * dz);
            const double* B = J + (int64_t)b * 4 * D.NV + v;
            const double x0 = x[2 * (int64_t)c], x1 = x[2 * (int64_t)c + 1];
            a0 += B[0] * x0 + B[D.NV] * x1;
            a1 += B[2 * (int64_t)D.NV] * x0 + B[3 * (int64_t)D.NV] * x1;
        }
        y[2 * (int64_t)v] = a0;
        y[2 * (int64_t)v + 1] = a1;
    }
}

// inverse of the diagonal blocks (block Jacobi, PreconditionerWrapperJacobi)
template <int DIM>
__global__ void kv_diag_inverse(VDims D, const double* __restrict__ J, double* __restrict__ dinv, int* flags) {
    constexpr int C = DIM == 3 ? 13 : 4;  // band of offset (0, 0, 0)
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < D.NV; v += gridDim.x * blockDim.x) {
        const double* B = J + (int64_t)C * 4 * D.NV + v;
        const double a = B[0], b = B[D.NV], c = B[2 * (int64_t)D.NV], d = B[3 * (int64_t)D.NV];
        const double det = a * d - b * c;
        if (det == 0.0 || !isfinite(det)) atomicOr(flags, 2);
        const double di = 1.0 / det;
        dinv[4 * (int64_t)v] = d * di;
        dinv[4 * (int64_t)v + 1] = -b * di;
        dinv[4 * (int64_t)v + 2] = -c * di;
        dinv[4 * (int64_t)v + 3] = a * di;
    }
}

// ---- block ILU(0) in the parity-colour order ------------------------------------------------------
//
// Vertices with the same parities (i & 1, j & 1, k & 1) never share an element, so ordering the
// vertices by that colour (then lexicographically) gives a block ILU(0) whose rows of one colour
// are independent: the factorisation and each triangular sweep run colour by colour, all vertices
// of a colour in parallel. It is dune-istl's bilu0 / bilu_backsolve (the factorisation the reference
// preconditioner runs, istlpreconditionerwrappers.hh:155-193) on the colour-permuted matrix; the
// stored diagonal block is its inverse.

struct VColour {
    int bx, by, bz;       // parity bits of the colour
    int cx, cy, cz;       // vertices of this colour per axis
    int count;
};

__device__ __forceinline__ int v_of_colour(const VDims& D, const VColour& C, int t, int& i, int& j, int& k) {
    const int ii = t % C.cx, jj = (t / C.cx) % C.cy, kk = t / (C.cx * C.cy);
    i = 2 * ii + C.bx;
    j = 2 * jj + C.by;
    k = 2 * kk + C.bz;
    return i + D.nvx * (j + D.nvy * k);
}

// colour of the neighbour at band b of a vertex of colour c
template <int DIM>
__device__ __forceinline__ int band_colour(int c, int b) {
    const int dx = b % 3 - 1, dy = (b / 3) % 3 - 1, dz = DIM == 3 ? b / 9 - 1 : 0;
    return c ^ ((dx != 0) | ((dy != 0) << 1) | ((dz != 0) << 2));
}
template <int DIM>
__device__ __forceinline__ bool band_in_grid(const VDims& D, int i, int j, int k, int b) {
    const int dx = b % 3 - 1, dy = (b / 3) % 3 - 1, dz = DIM == 3 ? b / 9 - 1 : 0;
    const int ii = i + dx, jj = j + dy, kk = k + dz;
    return ii >= 0 && jj >= 0 && kk >= 0 && ii < D.nvx && jj < D.nvy && kk < D.nvz;
}
template <int DIM>
__device__ __forceinline__ int band_offset(const VDims& D, int b) {
    const int dx = b % 3 - 1, dy = (b / 3) % 3 - 1, dz = DIM == 3 ? b / 9 - 1 : 0;
    return dx + D.nvx * (dy + D.nvy * dz);
}

__device__ __forceinline__ void blk_mul(const double* A, const double* B, double* o) {  // o = A B
    const double o0 = A[0] * B[0] + A[1] * B[2], o1 = A[0] * B[1] + A[1] * B[3];
    const double o2 = A[2] * B[0] + A[3] * B[2], o3 = A[2] * B[1] + A[3] * B[3];
    o[0] = o0; o[1] = o1; o[2] = o2; o[3] = o3;
}

// factorisation of the rows of colour c (the rows of lower colours are final)
template <int DIM>
__global__ void kv_ilu_factor(VDims D, VColour C, int c, const double* __restrict__ J, double* __restrict__ M, int* flags) {
    constexpr int NB = DIM == 3 ? 27 : 9;
    constexpr int CB = DIM == 3 ? 13 : 4;
    const int64_t NV = D.NV;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < C.count; t += gridDim.x * blockDim.x) {
        int i, j, k;
        const int v = v_of_colour(D, C, t, i, j, k);
        for (int q = 0; q < NB * 4; ++q) M[q * NV + v] = J[q * NV + v];
        // eliminate the couplings to lower colours, column order: colour, then index
        for (int kc = 0; kc < c; ++kc) {
            for (int b = 0; b < NB; ++b) {
                if (band_colour<DIM>(c, b) != kc || !band_in_grid<DIM>(D, i, j, k, b)) continue;
                const int kv = v + band_offset<DIM>(D, b);
                double Lb[4], Dk[4];
                for (int e = 0; e < 4; ++e) { Lb[e] = M[(b * 4 + e) * NV + v]; Dk[e] = M[(CB * 4 + e) * NV + kv]; }
                blk_mul(Lb, Dk, Lb);  // A_vk inv(A_kk)
                for (int e = 0; e < 4; ++e) M[(b * 4 + e) * NV + v] = Lb[e];
                const int dxk = b % 3 - 1, dyk = (b / 3) % 3 - 1, dzk = DIM == 3 ? b / 9 - 1 : 0;
                for (int b2 = 0; b2 < NB; ++b2) {
                    if (band_colour<DIM>(c, b2) <= kc || !band_in_grid<DIM>(D, i, j, k, b2)) continue;
                    // column j2 = v + o(b2) in row k: offset o(b2) - o(b) must be a neighbour offset
                    const int rx = b2 % 3 - 1 - dxk, ry = (b2 / 3) % 3 - 1 - dyk, rz = (DIM == 3 ? b2 / 9 - 1 : 0) - dzk;
                    if (rx < -1 || rx > 1 || ry < -1 || ry > 1 || rz < -1 || rz > 1) continue;
                    const int bk = (rx + 1) + 3 * (ry + 1) + (DIM == 3 ? 9 * (rz + 1) : 0);
                    double Akj[4], B[4];
                    for (int e = 0; e < 4; ++e) Akj[e] = M[(bk * 4 + e) * NV + kv];
                    blk_mul(Lb, Akj, B);
                    for (int e = 0; e < 4; ++e) M[(b2 * 4 + e) * NV + v] -= B[e];
                }
            }
        }
        // invert the diagonal block in place
        double a[4];
        for (int e = 0; e < 4; ++e) a[e] = M[(CB * 4 + e) * NV + v];
        const double det = a[0] * a[3] - a[1] * a[2];
        if (det == 0.0 || !isfinite(det)) atomicOr(flags, 2);
        const double di = 1.0 / det;
        M[(CB * 4 + 0) * NV + v] = a[3] * di;
        M[(CB * 4 + 1) * NV + v] = -a[1] * di;
        M[(CB * 4 + 2) * NV + v] = -a[2] * di;
        M[(CB * 4 + 3) * NV + v] = a[0] * di;
    }
}

// colour flip of the neighbour at band b: bit a set when the offset along axis a is odd
template <int DIM>
__host__ __device__ constexpr int band_flip(int b) {
    return ((b % 3) != 1) | (((b / 3) % 3 != 1) << 1) | ((DIM == 3 && b / 9 != 1) << 2);
}

// forward sweep of colour c: y_v = d_v - sum over lower colours L_vk y_k (bands in index order)
template <int DIM>
__global__ void kv_ilu_fwd(VDims D, VColour C, int c, const double* __restrict__ M, const double* __restrict__ d,
                           double* __restrict__ y) {
    constexpr int NB = DIM == 3 ? 27 : 9;
    const int64_t NV = D.NV;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < C.count; t += gridDim.x * blockDim.x) {
        int i, j, k;
        const int v = v_of_colour(D, C, t, i, j, k);
        double r0 = d[2 * (int64_t)v], r1 = d[2 * (int64_t)v + 1];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if ((c ^ band_flip<DIM>(b)) >= c || !band_in_grid<DIM>(D, i, j, k, b)) continue;
            const int kv = v + band_offset<DIM>(D, b);
            const double x0 = y[2 * (int64_t)kv], x1 = y[2 * (int64_t)kv + 1];
            const double* L = M + (int64_t)b * 4 * NV + v;
            r0 -= L[0] * x0 + L[NV] * x1;
            r1 -= L[2 * NV] * x0 + L[3 * NV] * x1;
        }
        y[2 * (int64_t)v] = r0;
        y[2 * (int64_t)v + 1] = r1;
    }
}

// backward sweep of colour c (in place): z_v = inv(U_vv) (y_v - sum over higher colours U_vj z_j)
template <int DIM>
__global__ void kv_ilu_bwd(VDims D, VColour C, int c, const double* __restrict__ M, double* __restrict__ z) {
    constexpr int NB = DIM == 3 ? 27 : 9;
    constexpr int CB = DIM == 3 ? 13 : 4;
    const int64_t NV = D.NV;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < C.count; t += gridDim.x * blockDim.x) {
        int i, j, k;
        const int v = v_of_colour(D, C, t, i, j, k);
        double r0 = z[2 * (int64_t)v], r1 = z[2 * (int64_t)v + 1];
#pragma unroll
        for (int b = NB - 1; b >= 0; --b) {
            if ((c ^ band_flip<DIM>(b)) <= c || !band_in_grid<DIM>(D, i, j, k, b)) continue;
            const int jv = v + band_offset<DIM>(D, b);
            const double x0 = z[2 * (int64_t)jv], x1 = z[2 * (int64_t)jv + 1];
            const double* U = M + (int64_t)b * 4 * NV + v;
            r0 -= U[0] * x0 + U[NV] * x1;
            r1 -= U[2 * NV] * x0 + U[3 * NV] * x1;
        }
        const double* Di = M + (int64_t)CB * 4 * NV + v;
        z[2 * (int64_t)v] = Di[0] * r0 + Di[NV] * r1;
        z[2 * (int64_t)v + 1] = Di[2 * NV] * r0 + Di[3 * NV] * r1;
    }
}

__global__ void kv_scale(int64_t n, double w, double* __restrict__ x) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        x[q] *= w;
}

__global__ void kv_jacobi(int NV, double w, const double* __restrict__ dinv, const double* __restrict__ d,
                          double* __restrict__ out) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < NV; v += gridDim.x * blockDim.x) {
        const double* M = dinv + 4 * (int64_t)v;
        const double d0 = d[2 * (int64_t)v], d1 = d[2 * (int64_t)v + 1];
        out[2 * (int64_t)v] = w * (M[0] * d0 + M[1] * d1);
        out[2 * (int64_t)v + 1] = w * (M[2] * d0 + M[3] * d1);
    }
}

// per-block partial sums of up to two dot products and two max-norms, in a fixed grid order
constexpr int kVRedBlocks = 296;
__global__ void __launch_bounds__(kVApi) kv_reduce(int64_t n, const double* __restrict__ a0, const double* __restrict__ b0,
                                                   const double* __restrict__ a1, const double* __restrict__ b1,
                                                   const double* __restrict__ m, const double* __restrict__ m2,
                                                   double* __restrict__ part) {
    double s0 = 0.0, s1 = 0.0, mx = 0.0, mx2 = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        if (a0) s0 += a0[q] * b0[q];
        if (a1) s1 += a1[q] * b1[q];
        if (m) mx = fmax(mx, fabs(m[q]));
        if (m2) mx2 = fmax(mx2, fabs(m2[q]));
    }
    __shared__ double sh[4][kVApi / 32];
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mx2 = fmax(mx2, __shfl_xor_sync(0xffffffffu, mx2, o));
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[0][w] = s0; sh[1][w] = s1; sh[2][w] = mx; sh[3][w] = mx2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        for (int q = 0; q < kVApi / 32; ++q) {
            t0 += sh[0][q]; t1 += sh[1][q]; t2 = fmax(t2, sh[2][q]); t3 = fmax(t3, sh[3][q]);
        }
        part[4 * blockIdx.x] = t0;
        part[4 * blockIdx.x + 1] = t1;
        part[4 * blockIdx.x + 2] = t2;
        part[4 * blockIdx.x + 3] = t3;
    }
}
__global__ void kv_reduce_final(int nblocks, const double* __restrict__ part, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        for (int q = 0; q < nblocks; ++q) {
            t0 += part[4 * q]; t1 += part[4 * q + 1]; t2 = fmax(t2, part[4 * q + 2]); t3 = fmax(t3, part[4 * q + 3]);
        }
        out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
    }
}

// vector updates of BiCGStabSolver::apply (bicgstabsolver.hh:191-322) with host-side scalars
__global__ void kv_p_update(int64_t n, double omega, double beta, const double* __restrict__ r,
                            const double* __restrict__ v, double* __restrict__ p) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        double tmp = v[q];
        tmp *= omega;
        tmp -= p[q];
        tmp *= -beta;
        p[q] = r[q] + tmp;
    }
}
__global__ void kv_h_s(int64_t n, double alpha, const double* __restrict__ y, const double* __restrict__ v,
                       double* __restrict__ x, double* __restrict__ r) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        x[q] = y[q] * alpha + x[q];
        r[q] -= v[q] * alpha;
    }
}
__global__ void kv_axpy(int64_t n, double a, const double* __restrict__ z, double* __restrict__ x) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        x[q] += a * z[q];
}
__global__ void kv_residual(int64_t n, const double* __restrict__ b, const double* __restrict__ ax, double* __restrict__ r) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        r[q] = b[q] - ax[q];
}
__global__ void kv_sub_update(int NV, const double2* __restrict__ dx, double2* __restrict__ x) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < NV; v += gridDim.x * blockDim.x) {
        const double2 a = x[v], d = dx[v];
        x[v] = make_double2(a.x - d.x, a.y - d.y);
    }
}

}  // namespace ewg

using namespace ewg;

namespace {

int vgrid(const ewg_vcfv* c, int64_t n, int block = kVApi) {
    int64_t need = (n + block - 1) / block;
    int64_t cap = (int64_t)c->numSMs * 8;
    return (int)(need < cap ? (need > 0 ? need : 1) : cap);
}

ewg_status vcheck(ewg_vcfv* c, const char* what) {
    ++c->launches;
    return vfail(c, cudaGetLastError(), what);
}

ewg_status v_storage(ewg_vcfv* c) {
    kv_storage<<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->P, c->x1, c->sold);
    return vcheck(c, "kv_storage");
}

// one pass of kv_reduce: a0.b0, a1.b1, max|m| and max|m2|; synchronous read-back of the four
ewg_status v_reduce(ewg_vcfv* c, const double* a0, const double* b0, const double* a1, const double* b1,
                    const double* m, const double* m2, double out[4]) {
    const int64_t n = 2 * (int64_t)c->D.NV;
    kv_reduce<<<kVRedBlocks, kVApi, 0, c->stream>>>(n, a0, b0, a1, b1, m, m2, c->s_red);
    ewg_status st = vcheck(c, "kv_reduce");
    if (st) return st;
    kv_reduce_final<<<1, 32, 0, c->stream>>>(kVRedBlocks, c->s_red, c->s_red + 4 * kVRedBlocks);
    if ((st = vcheck(c, "kv_reduce_final"))) return st;
    cudaError_t e = cudaMemcpyAsync(c->h_red, c->s_red + 4 * kVRedBlocks, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return vfail(c, e, "reduce read-back");
    for (int q = 0; q < 4; ++q) out[q] = c->h_red[q];
    return EWG_OK;
}

ewg_status v_spmv(ewg_vcfv* c, const double* x, double* y) {
    if (c->P.dim == 3) kv_spmv<3><<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->D, c->J, x, y);
    else kv_spmv<2><<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->D, c->J, x, y);
    return vcheck(c, "kv_spmv");
}

VColour v_colour(const ewg_vcfv* c, int col) {
    VColour C;
    C.bx = col & 1; C.by = (col >> 1) & 1; C.bz = (col >> 2) & 1;
    C.cx = (c->D.nvx - C.bx + 1) / 2;
    C.cy = (c->D.nvy - C.by + 1) / 2;
    C.cz = (c->D.nvz - C.bz + 1) / 2;
    C.count = C.cx * C.cy * C.cz;
    return C;
}
int v_ncolours(const ewg_vcfv* c) { return c->P.dim == 3 ? 8 : 4; }

// block ILU(0) factorisation of J in the parity-colour order, colour by colour
ewg_status v_ilu_factor(ewg_vcfv* c) {
    if (!c->M) {
        cudaError_t e = cudaMalloc(&c->M, sizeof(double) * c->nb * 4 * (size_t)c->D.NV);
        if (e != cudaSuccess) return vfail(c, e, "alloc ILU factors");
        if ((e = cudaMemsetAsync(c->M, 0, sizeof(double) * c->nb * 4 * (size_t)c->D.NV, c->stream)) != cudaSuccess)
            return vfail(c, e, "zero ILU factors");
    }
    for (int col = 0; col < v_ncolours(c); ++col) {
        const VColour C = v_colour(c, col);
        if (C.count == 0) continue;
        if (c->P.dim == 3) kv_ilu_factor<3><<<vgrid(c, C.count), kVApi, 0, c->stream>>>(c->D, C, col, c->J, c->M, c->d_flags);
        else kv_ilu_factor<2><<<vgrid(c, C.count), kVApi, 0, c->stream>>>(c->D, C, col, c->J, c->M, c->d_flags);
        ewg_status st = vcheck(c, "kv_ilu_factor");
        if (st) return st;
    }
    return EWG_OK;
}

// the ILU(0) application as direct launches on the context's stream
ewg_status v_ilu_apply(ewg_vcfv* c, double w, const double* d, double* out) {
    const int nc = v_ncolours(c);
    for (int col = 0; col < nc; ++col) {
        const VColour C = v_colour(c, col);
        if (C.count == 0) continue;
        if (c->P.dim == 3) kv_ilu_fwd<3><<<vgrid(c, C.count), kVApi, 0, c->stream>>>(c->D, C, col, c->M, d, out);
        else kv_ilu_fwd<2><<<vgrid(c, C.count), kVApi, 0, c->stream>>>(c->D, C, col, c->M, d, out);
        ewg_status st = vcheck(c, "kv_ilu_fwd");
        if (st) return st;
    }
    for (int col = nc - 1; col >= 0; --col) {
        const VColour C = v_colour(c, col);
        if (C.count == 0) continue;
        if (c->P.dim == 3) kv_ilu_bwd<3><<<vgrid(c, C.count), kVApi, 0, c->stream>>>(c->D, C, col, c->M, out);
        else kv_ilu_bwd<2><<<vgrid(c, C.count), kVApi, 0, c->stream>>>(c->D, C, col, c->M, out);
        ewg_status st = vcheck(c, "kv_ilu_bwd");
        if (st) return st;
    }
    if (w != 1.0) {
        kv_scale<<<vgrid(c, 2 * (int64_t)c->D.NV), kVApi, 0, c->stream>>>(2 * (int64_t)c->D.NV, w, out);
        return vcheck(c, "kv_scale");
    }
    return EWG_OK;
}

// y = M^-1 d. Block ILU(0) replays a CUDA graph of its 2 x (colours) sweep launches: the
// factors, colour tables and vectors keep their addresses for the context's lifetime, so a graph
// captured for (d, out, w) stays valid; the first application of a pair captures it.
ewg_status v_prec(ewg_vcfv* c, double w, const double* d, double* out) {
    if (c->precond != EWG_PRECOND_ILU0) {
        kv_jacobi<<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->D.NV, w, c->s_dinv, d, out);
        return vcheck(c, "kv_jacobi");
    }
    for (auto& g : c->precGraphs) {
        if (g.exec && g.d == d && g.out == out && g.w == w) {
            c->launches += g.kernels;
            return vfail(c, cudaGraphLaunch(g.exec, c->stream), "ILU graph launch");
        }
    }
    ewg_vcfv::PrecGraph* slot = nullptr;
    for (auto& g : c->precGraphs) if (!g.exec) { slot = &g; break; }
    if (!slot) {
        slot = &c->precGraphs[c->precGraphNext];
        c->precGraphNext ^= 1;
        cudaGraphExecDestroy(slot->exec);
        slot->exec = nullptr;
    }
    const long long before = c->launches;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return vfail(c, e, "ILU graph capture");
    ewg_status st = v_ilu_apply(c, w, d, out);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(c->stream, &graph);
    const int kernels = (int)(c->launches - before);
    c->launches = before;
    if (st || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return st ? st : vfail(c, e, "ILU graph capture");
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return vfail(c, e, "ILU graph instantiate");
    slot->d = d;
    slot->out = out;
    slot->w = w;
    slot->kernels = kernels;
    slot->exec = exec;
    c->launches += kernels;
    return vfail(c, cudaGraphLaunch(exec, c->stream), "ILU graph launch");
}

}  // namespace

extern "C" {

ewg_status ewg_vcfv_create(const ewg_grid* grid, const ewg_problem* problem, const double* perm, ewg_vcfv** out) {
    if (!grid || !problem || !perm || !out) return EWG_ERR_INVALID;
    *out = nullptr;
    if (grid->dim != 2 && grid->dim != 3) return EWG_ERR_INVALID;
    const int nz = grid->dim == 3 ? grid->nz : 1;
    if (grid->nx < 1 || grid->ny < 1 || nz < 1) return EWG_ERR_INVALID;
    if (grid->dim == 3 && grid->k_origin != 0) return EWG_ERR_INVALID;  // whole grids only
    const int64_t nv = (int64_t)(grid->nx + 1) * (grid->ny + 1) * (grid->dim == 3 ? nz + 1 : 1);
    if (nv * (grid->dim == 3 ? 27 : 9) * 4 >= ((int64_t)1 << 40) || nv >= ((int64_t)1 << 31) / 2)
        return EWG_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) { cudaGetLastError(); return EWG_ERR_NO_DEVICE; }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10) return EWG_ERR_NO_DEVICE;
    ewg_vcfv* c = new ewg_vcfv();
    c->device = dev;
    c->numSMs = prop.multiProcessorCount;
    build_phys(c->P, grid, problem);
    c->P.N = nv;  // plane stride of the intensive-quantity cache
    c->D.nvx = grid->nx + 1;
    c->D.nvy = grid->ny + 1;
    c->D.nvz = grid->dim == 3 ? nz + 1 : 1;
    c->D.nex = grid->nx;
    c->D.ney = grid->ny;
    c->D.nez = nz;
    c->D.NV = (int)nv;
    c->nb = grid->dim == 3 ? 27 : 9;
    c->hgeo = build_vgeom(c->P);
    auto fail = [&](cudaError_t e, const char* what) {
        c->err = std::string(what) + ": " + cudaGetErrorString(e);
        return EWG_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) { ewg_status s = fail(e, "stream"); delete c; return s; }
    const size_t v2 = sizeof(double2) * nv, v1 = sizeof(double) * nv;
    struct A { void** p; size_t n; } allocs[] = {
        {(void**)&c->x0, v2}, {(void**)&c->x1, v2}, {(void**)&c->sold, v2}, {(void**)&c->r, v2},
        {(void**)&c->perm, v1}, {(void**)&c->totVol, v1}, {(void**)&c->iq, 6 * v1}, {(void**)&c->kedge, 3 * v1},
        {(void**)&c->J, (size_t)c->nb * 4 * v1}, {(void**)&c->lens, (size_t)nv}, {(void**)&c->geo, sizeof(VGeomDev)},
        {(void**)&c->d_errmax, sizeof(unsigned long long)}, {(void**)&c->d_flags, sizeof(int)},
        {(void**)&c->s_b, v2}, {(void**)&c->s_x, v2}, {(void**)&c->s_r, v2}, {(void**)&c->s_r0, v2},
        {(void**)&c->s_v, v2}, {(void**)&c->s_p, v2}, {(void**)&c->s_y, v2}, {(void**)&c->s_z, v2},
        {(void**)&c->s_t, v2}, {(void**)&c->s_dinv, 2 * v2}, {(void**)&c->s_red, sizeof(double) * (4 * kVRedBlocks + 4)}};
    for (auto& a : allocs)
        if ((e = cudaMalloc(a.p, a.n)) != cudaSuccess) { ewg_status s = fail(e, "device allocation"); ewg_vcfv_destroy(c); return s; }
    if ((e = cudaMallocHost(&c->h_red, 4 * sizeof(double))) != cudaSuccess) { ewg_status s = fail(e, "pinned"); ewg_vcfv_destroy(c); return s; }
    // vertex lens flags from the vertex positions (isInLens_)
    std::vector<uint8_t> lensH(nv);
    for (int64_t v = 0; v < nv; ++v) {
        const int64_t id[3] = {v % c->D.nvx, (v / c->D.nvx) % c->D.nvy, v / ((int64_t)c->D.nvx * c->D.nvy)};
        double xv[3];
        for (int d = 0; d < 3; ++d) xv[d] = d < grid->dim ? id[d] * c->P.h[d] : 0.0;
        bool in = true;
        for (int a = 0; a < grid->dim; ++a)
            if (xv[a] < problem->lens_lo[a] - problem->eps || xv[a] > problem->lens_hi[a] + problem->eps) in = false;
        lensH[v] = in ? 1 : 0;
    }
    if ((e = cudaMemcpyAsync(c->perm, perm, v1, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->lens, lensH.data(), nv, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->geo, &c->hgeo, sizeof(VGeomDev), cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->J, 0, (size_t)c->nb * 4 * v1, c->stream)) != cudaSuccess) {
        ewg_status s = fail(e, "upload"); ewg_vcfv_destroy(c); return s;
    }
    kv_total_volume<<<vgrid(c, nv), kVApi, 0, c->stream>>>(c->D, grid->dim, c->hgeo.scvVol, c->totVol);
    kv_edge_perm<<<vgrid(c, nv), kVApi, 0, c->stream>>>(c->D, grid->dim, c->perm, c->kedge);
    if ((e = cudaGetLastError()) != cudaSuccess) { ewg_status s = fail(e, "total volume"); ewg_vcfv_destroy(c); return s; }
    if ((e = boundary_constants(c->P, c->stream)) != cudaSuccess) { ewg_status s = fail(e, "boundary constants"); ewg_vcfv_destroy(c); return s; }
    const int smem = (int)(sizeof(double) * (grid->dim == 3 ? vcfv_slots<3>() : vcfv_slots<2>()) * 4 * kVBlock);
    e = grid->dim == 3 ? cudaFuncSetAttribute(kv_assemble<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                       : cudaFuncSetAttribute(kv_assemble<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = grid->dim == 3 ? cudaFuncSetAttribute(kv_assemble<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                           : cudaFuncSetAttribute(kv_assemble<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess || (e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
        ewg_status s = fail(e, "setup"); ewg_vcfv_destroy(c); return s;
    }
    *out = c;
    return EWG_OK;
}

void ewg_vcfv_destroy(ewg_vcfv* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& g : c->precGraphs) if (g.exec) cudaGraphExecDestroy(g.exec);
    void* ps[] = {c->x0, c->x1, c->sold, c->r, c->perm, c->totVol, c->kedge, c->iq, c->J, c->lens, c->geo, c->d_errmax,
                  c->d_flags, c->s_b, c->s_x, c->s_r, c->s_r0, c->s_v, c->s_p, c->s_y, c->s_z, c->s_t, c->s_dinv,
                  c->s_red, c->M};
    for (void* p : ps) if (p) cudaFree(p);
    if (c->h_red) cudaFreeHost(c->h_red);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* ewg_vcfv_last_error(const ewg_vcfv* c) { return c ? c->err.c_str() : "null context"; }
int64_t ewg_vcfv_num_dofs(const ewg_vcfv* c) { return c ? c->D.NV : 0; }
int64_t ewg_vcfv_launches(const ewg_vcfv* c) { return c ? c->launches : 0; }

ewg_status ewg_vcfv_set_solution(ewg_vcfv* c, int32_t timeIdx, const double* x) {
    if (!c || !x || (timeIdx != 0 && timeIdx != 1)) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(timeIdx == 0 ? c->x0 : c->x1, x, sizeof(double2) * c->D.NV, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return vfail(c, e, "set solution");
    if (timeIdx == 1) { ewg_status st = v_storage(c); if (st) return st; }
    return vfail(c, cudaStreamSynchronize(c->stream), "set solution");
}

ewg_status ewg_vcfv_get_solution(ewg_vcfv* c, int32_t timeIdx, double* x) {
    if (!c || !x || (timeIdx != 0 && timeIdx != 1)) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(x, timeIdx == 0 ? c->x0 : c->x1, sizeof(double2) * c->D.NV, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return vfail(c, e, "get solution");
}

ewg_status ewg_vcfv_apply_initial_solution(ewg_vcfv* c) {
    if (!c) return EWG_ERR_INVALID;
    kv_initial<<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->P, c->D, c->x0);
    ewg_status st = vcheck(c, "kv_initial");
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(c->x1, c->x0, sizeof(double2) * c->D.NV, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return vfail(c, e, "initial copy");
    if ((st = v_storage(c))) return st;
    return vfail(c, cudaStreamSynchronize(c->stream), "initial solution");
}

ewg_status ewg_vcfv_advance_time_level(ewg_vcfv* c) {
    if (!c) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(c->x1, c->x0, sizeof(double2) * c->D.NV, cudaMemcpyDeviceToDevice, c->stream);
    if (e != cudaSuccess) return vfail(c, e, "advance");
    ewg_status st = v_storage(c);
    if (st) return st;
    return vfail(c, cudaStreamSynchronize(c->stream), "advance");
}

ewg_status ewg_vcfv_restore_time_level(ewg_vcfv* c) {
    if (!c) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(c->x0, c->x1, sizeof(double2) * c->D.NV, cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return vfail(c, e, "restore");
}

ewg_status ewg_vcfv_set_local_linearizer(ewg_vcfv* c, int32_t kind, int32_t method) {
    if (!c) return EWG_ERR_INVALID;
    if (kind != EWG_LOCAL_LINEARIZER_AD && kind != EWG_LOCAL_LINEARIZER_FD) { c->err = "unknown local linearizer"; return EWG_ERR_INVALID; }
    if (method < -1 || method > 1) { c->err = "NumericDifferenceMethod must be -1, 0 or +1"; return EWG_ERR_INVALID; }
    c->localLinearizer = kind;
    c->fdMethod = method;
    return EWG_OK;
}

ewg_status ewg_vcfv_update_begin(ewg_vcfv* c) {
    if (!c) return EWG_ERR_INVALID;
    double2 v0;
    cudaError_t e = cudaMemcpyAsync(&v0, c->x0, sizeof(double2), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return vfail(c, e, "update begin");
    c->refPressure = v0.x;
    return EWG_OK;
}

// residual (volumetric) and Jacobian of solution(0); *error = max |r|, NaN/Inf -> EWG_ERR_NONFINITE
ewg_status ewg_vcfv_linearize(ewg_vcfv* c, double dt, double* error) {
    if (!c || !(dt > 0)) return EWG_ERR_INVALID;
    cudaError_t e;
    if ((e = cudaMemsetAsync(c->d_errmax, 0, sizeof(unsigned long long), c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->d_flags, 0, sizeof(int), c->stream)) != cudaSuccess)
        return vfail(c, e, "memset");
    kv_intensive<<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->P, c->x0, c->lens, c->iq);
    ewg_status st = vcheck(c, "kv_intensive");
    if (st) return st;
    const int blocks = (c->D.NV + kVBlock - 1) / kVBlock;
    const size_t smem = sizeof(double) * (c->P.dim == 3 ? vcfv_slots<3>() : vcfv_slots<2>()) * 4 * kVBlock;
    const bool fd = c->localLinearizer == EWG_LOCAL_LINEARIZER_FD;
    if (fd && !(c->refPressure > 0)) {
        // a context that never ran updateBegin takes the reference pressure of the current iterate
        if ((st = ewg_vcfv_update_begin(c))) return st;
    }
    auto k = c->P.dim == 3 ? (fd ? kv_assemble<3, true> : kv_assemble<3, false>)
                           : (fd ? kv_assemble<2, true> : kv_assemble<2, false>);
    k<<<blocks, kVBlock, smem, c->stream>>>(c->P, c->D, c->geo, c->x0, c->sold, c->perm, c->lens, c->iq, c->kedge,
                                            c->totVol, dt, c->refPressure, c->fdMethod, c->r, c->J, c->d_errmax,
                                            c->d_flags);
    if ((st = vcheck(c, "kv_assemble"))) return st;
    unsigned long long bits = 0;
    int flag = 0;
    if ((e = cudaMemcpyAsync(&bits, c->d_errmax, sizeof(bits), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&flag, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return vfail(c, e, "linearize read-back");
    double v;
    memcpy(&v, &bits, sizeof(v));
    if (error) *error = flag ? INFINITY : v;
    if (flag) { c->err = "non-finite residual"; return EWG_ERR_NONFINITE; }
    return EWG_OK;
}

ewg_status ewg_vcfv_get_residual(ewg_vcfv* c, double* r) {
    if (!c || !r) return EWG_ERR_INVALID;
    cudaError_t e = cudaMemcpyAsync(r, c->r, sizeof(double2) * c->D.NV, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return vfail(c, e, "get residual");
}

// the Jacobian in BCRS with the caller's natural pattern (row_ptr / col_idx of the vertex stencil)
ewg_status ewg_vcfv_get_jacobian_bcrs(ewg_vcfv* c, const int32_t* rowPtr, const int32_t* colIdx, int64_t nnzb,
                                      double* blocks) {
    if (!c || !rowPtr || !colIdx || !blocks) return EWG_ERR_INVALID;
    // every block must be a stored band: the column a vertex of the row's 3x3(x3) neighbourhood
    if (rowPtr[0] != 0 || rowPtr[c->D.NV] != nnzb) { c->err = "row pointers do not span nnzb blocks"; return EWG_ERR_INVALID; }
    for (int v = 0; v < c->D.NV; ++v) {
        if (rowPtr[v + 1] < rowPtr[v]) { c->err = "row pointers decrease"; return EWG_ERR_INVALID; }
        const int i = v % c->D.nvx, j = (v / c->D.nvx) % c->D.nvy, k = v / (c->D.nvx * c->D.nvy);
        for (int32_t q = rowPtr[v]; q < rowPtr[v + 1]; ++q) {
            const int col = colIdx[q];
            if (col < 0 || col >= c->D.NV) { c->err = "column index out of range"; return EWG_ERR_INVALID; }
            const int ci = col % c->D.nvx, cj = (col / c->D.nvx) % c->D.nvy, ck = col / (c->D.nvx * c->D.nvy);
            if (std::abs(ci - i) > 1 || std::abs(cj - j) > 1 || std::abs(ck - k) > 1) {
                c->err = "the pattern holds a block outside the vertex stencil";
                return EWG_ERR_INVALID;
            }
        }
    }
    int32_t *dr = nullptr, *dc = nullptr;
    double* db = nullptr;
    cudaError_t e = cudaMalloc(&dr, sizeof(int32_t) * (c->D.NV + 1));
    if (e == cudaSuccess) e = cudaMalloc(&dc, sizeof(int32_t) * nnzb);
    if (e == cudaSuccess) e = cudaMalloc(&db, sizeof(double) * 4 * nnzb);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dr, rowPtr, sizeof(int32_t) * (c->D.NV + 1), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, colIdx, sizeof(int32_t) * nnzb, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        kv_to_bcrs<<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->D, c->P.dim, c->J, dr, dc, db);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(blocks, db, sizeof(double) * 4 * nnzb, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (dr) cudaFree(dr);
    if (dc) cudaFree(dc);
    if (db) cudaFree(db);
    return vfail(c, e, "jacobian export");
}

// BiCGStabSolver::apply (bicgstabsolver.hh:116-326) on J dx = r with block Jacobi, the
// CombinedCriterion (combinedcriterion.hh:112-205) and the shadow-residual restart / true-residual
// check options of ewg_solve_opts; dx stays on the device (the Newton update reads it)
static ewg_status vcfv_solve(ewg_vcfv* c, const ewg_solve_opts* so, int* iterations) {
    const int64_t n = 2 * (int64_t)c->D.NV;
    const int g = vgrid(c, n);
    cudaStream_t s = c->stream;
    ewg_status st;
    *iterations = 0;
    cudaError_t e;
    if ((e = cudaMemsetAsync(c->d_flags, 0, sizeof(int), s)) != cudaSuccess) return vfail(c, e, "memset");
    c->precond = so->precond;
    if (so->precond == EWG_PRECOND_ILU0) {
        if ((st = v_ilu_factor(c))) return st;
    } else {
        if (c->P.dim == 3) kv_diag_inverse<3><<<vgrid(c, c->D.NV), kVApi, 0, s>>>(c->D, c->J, c->s_dinv, c->d_flags);
        else kv_diag_inverse<2><<<vgrid(c, c->D.NV), kVApi, 0, s>>>(c->D, c->J, c->s_dinv, c->d_flags);
        if ((st = vcheck(c, "kv_diag_inverse"))) return st;
    }
    // b = r, x = 0, r = b, r0hat = b
    if ((e = cudaMemcpyAsync(c->s_b, c->r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->s_r, c->r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->s_r0, c->r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->s_x, 0, sizeof(double) * n, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->s_v, 0, sizeof(double) * n, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->s_p, 0, sizeof(double) * n, s)) != cudaSuccess)
        return vfail(c, e, "solver init");
    double red[4];
    if ((st = v_reduce(c, c->s_r0, c->s_r0, nullptr, nullptr, c->s_r, nullptr, red))) return st;
    int sing = 0;
    if ((e = cudaMemcpyAsync(&sing, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return vfail(c, e, "flags");
    if (sing & 2) { c->err = "singular diagonal block"; return EWG_ERR_BREAKDOWN; }
    const double breakdownEps = 2.2250738585072014e-308 * 1e10;
    double r0r0 = red[0];
    double resErr = fmax(red[2], breakdownEps);
    const double initResErr = resErr;
    auto converged = [&](double err) { return err / fmax(1e-20, initResErr) <= so->linear_solver_tolerance ||
                                              err <= so->linear_solver_abs_tolerance; };
    if (converged(resErr)) {
        return vfail(c, cudaMemsetAsync(c->s_x, 0, sizeof(double) * n, s), "zero update");
    }
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int replacements = 0;
    const double w = so->preconditioner_relaxation;
    // true-residual check on convergence: true when the iteration must go on
    auto replace = [&](bool* goOn) -> ewg_status {
        *goOn = false;
        if (!so->verify_true_residual || replacements >= 3) return EWG_OK;
        ewg_status q = v_spmv(c, c->s_x, c->s_t);
        if (q) return q;
        kv_residual<<<g, kVApi, 0, s>>>(n, c->s_b, c->s_t, c->s_r);
        if ((q = vcheck(c, "kv_residual"))) return q;
        double rr[4];
        if ((q = v_reduce(c, c->s_r, c->s_r, nullptr, nullptr, c->s_r, nullptr, rr))) return q;
        if (rr[2] / fmax(1e-20, initResErr) <= 10 * so->linear_solver_tolerance ||
            rr[2] <= 10 * so->linear_solver_abs_tolerance)
            return EWG_OK;
        ++replacements;
        cudaError_t ee = cudaMemcpyAsync(c->s_r0, c->s_r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        if (ee == cudaSuccess) ee = cudaMemsetAsync(c->s_v, 0, sizeof(double) * n, s);
        if (ee == cudaSuccess) ee = cudaMemsetAsync(c->s_p, 0, sizeof(double) * n, s);
        if (ee != cudaSuccess) return vfail(c, ee, "replace");
        r0r0 = rr[0];
        rho = alpha = omega = 1.0;
        resErr = rr[2];
        *goOn = true;
        return EWG_OK;
    };
    const int maxIt = so->linear_solver_max_iterations;
    int it = 0;
    for (; it < maxIt; ++it) {
        double rr[4];
        // rho_i = r0hat . r, |r|^2
        if ((st = v_reduce(c, c->s_r0, c->s_r, c->s_r, c->s_r, nullptr, nullptr, rr))) return st;
        double rho_i = rr[0];
        if (so->restart_on_breakdown && fabs(rho_i) <= 1e-12 * sqrt(r0r0) * sqrt(rr[1])) {
            if ((e = cudaMemcpyAsync(c->s_r0, c->s_r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s)) != cudaSuccess ||
                (e = cudaMemsetAsync(c->s_v, 0, sizeof(double) * n, s)) != cudaSuccess ||
                (e = cudaMemsetAsync(c->s_p, 0, sizeof(double) * n, s)) != cudaSuccess)
                return vfail(c, e, "restart");
            r0r0 = rr[1];
            rho_i = rr[1];
            rho = alpha = omega = 1.0;
        }
        if (fabs(rho) <= breakdownEps || fabs(omega) <= breakdownEps) { c->err = "BiCGStab breakdown"; return EWG_ERR_BREAKDOWN; }
        const double beta = (rho_i / rho) * (alpha / omega);
        rho = rho_i;
        kv_p_update<<<g, kVApi, 0, s>>>(n, omega, beta, c->s_r, c->s_v, c->s_p);
        if ((st = vcheck(c, "kv_p_update"))) return st;
        if ((st = v_prec(c, w, c->s_p, c->s_y))) return st;
        if ((st = v_spmv(c, c->s_y, c->s_v))) return st;
        // r0hat . v, and max |y|: the update y stagnates when it is all zero
        if ((st = v_reduce(c, c->s_r0, c->s_v, nullptr, nullptr, c->s_y, nullptr, rr))) return st;
        const bool stagY = rr[2] == 0.0;
        if (fabs(rr[0]) <= breakdownEps) { c->err = "BiCGStab breakdown"; return EWG_ERR_BREAKDOWN; }
        alpha = rho_i / rr[0];
        if (fabs(alpha) <= breakdownEps) { c->err = "BiCGStab stagnation"; return EWG_ERR_BREAKDOWN; }
        kv_h_s<<<g, kVApi, 0, s>>>(n, alpha, c->s_y, c->s_v, c->s_x, c->s_r);
        if ((st = vcheck(c, "kv_h_s"))) return st;
        // z = M^-1 s and t = J z come before the half-step check, so that max |s| for the
        // criterion shares one read-back with t.t, t.s and max |z|; when the half step ends the
        // solve (or replaces the residual), z and t are left unused
        if ((st = v_prec(c, w, c->s_r, c->s_z))) return st;
        if ((st = v_spmv(c, c->s_z, c->s_t))) return st;
        if ((st = v_reduce(c, c->s_t, c->s_t, c->s_t, c->s_r, c->s_r, c->s_z, rr))) return st;
        resErr = rr[2];
        if (converged(resErr)) {
            bool goOn;
            if ((st = replace(&goOn))) return st;
            if (!goOn) { *iterations = it; return EWG_OK; }
            continue;
        }
        if (stagY || resErr > so->linear_solver_max_error) { *iterations = it; c->err = "BiCGStab failed"; return EWG_ERR_NOT_CONVERGED; }
        if (fabs(rr[0]) <= breakdownEps) { c->err = "BiCGStab breakdown"; return EWG_ERR_BREAKDOWN; }
        omega = rr[1] / rr[0];
        if (fabs(omega) <= breakdownEps) { c->err = "BiCGStab stagnation"; return EWG_ERR_BREAKDOWN; }
        kv_axpy<<<g, kVApi, 0, s>>>(n, omega, c->s_z, c->s_x);
        if ((st = vcheck(c, "kv_axpy"))) return st;
        // the criterion sees s (the reference's aliasing r == s) before r = s - omega t; the
        // update z stagnates when it is all zero
        const bool stag = rr[3] == 0.0;
        if (converged(resErr)) {
            bool goOn;
            if ((st = replace(&goOn))) return st;
            if (!goOn) { *iterations = it; return EWG_OK; }
            continue;
        }
        if (stag || resErr > so->linear_solver_max_error) { *iterations = it; c->err = "BiCGStab failed"; return EWG_ERR_NOT_CONVERGED; }
        kv_axpy<<<g, kVApi, 0, s>>>(n, -omega, c->s_t, c->s_r);
        if ((st = vcheck(c, "kv_axpy"))) return st;
    }
    *iterations = it;
    c->err = "BiCGStab: maximum iterations";
    return EWG_ERR_NOT_CONVERGED;
}

// ParallelBaseBackend::solve (parallelbasebackend.hh:301-338) on the last linearization: the
// update dx with J dx = r (dx_out nullable: the update stays on the device)
ewg_status ewg_vcfv_solve(ewg_vcfv* c, const ewg_solve_opts* so, double* dx_out, int32_t* iterations) {
    if (!c || !so) return EWG_ERR_INVALID;
    if (so->precond != EWG_PRECOND_JACOBI && so->precond != EWG_PRECOND_ILU0) { c->err = "unknown preconditioner"; return EWG_ERR_INVALID; }
    if (so->precision != EWG_PRECISION_FP64) { c->err = "the vertex-centred solve is FP64"; return EWG_ERR_INVALID; }
    int it = 0;
    ewg_status st = vcfv_solve(c, so, &it);
    if (iterations) *iterations = it;
    if (st) return st;
    if (dx_out) {
        cudaError_t e = cudaMemcpyAsync(dx_out, c->s_x, sizeof(double2) * c->D.NV, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        return vfail(c, e, "get update");
    }
    return EWG_OK;
}

// NewtonMethod::apply at fixed dt (newtonmethod.hh:308-517): linearize, convergence test on the
// residual max-norm before the solve, BiCGStab + block Jacobi, x -= dx
ewg_status ewg_vcfv_newton_apply(ewg_vcfv* c, double dt, const ewg_newton_opts* no, const ewg_solve_opts* so,
                                 int32_t* newtonIts, int32_t* linIts, double* errorOut) {
    if (!c || !no || !so || !(dt > 0)) return EWG_ERR_INVALID;
    if (so->precond != EWG_PRECOND_JACOBI && so->precond != EWG_PRECOND_ILU0) { c->err = "unknown preconditioner"; return EWG_ERR_INVALID; }
    if (so->precision != EWG_PRECISION_FP64) { c->err = "the vertex-centred solve is FP64"; return EWG_ERR_INVALID; }
    int numIterations = 0, linTotal = 0;
    double error = 1e100, lastError = 1e100;
    auto converged = [&]() { return error <= no->newton_tolerance; };
    auto proceed = [&]() {
        if (numIterations < 1) return true;
        if (converged()) return false;
        if (numIterations >= no->newton_max_iterations) return error * 4.0 < lastError;
        return true;
    };
    // ImmiscibleModel::updateBegin before every Newton solve
    ewg_status status = ewg_vcfv_update_begin(c);
    if (status) return status;
    while (proceed()) {
        double err = 0.0;
        ewg_status st = ewg_vcfv_linearize(c, dt, &err);
        if (st) { status = st; break; }
        lastError = error;
        error = err;
        if (error > no->newton_max_error) { status = EWG_ERR_MAX_ERROR; c->err = "Newton: error above NewtonMaxError"; break; }
        if (!proceed()) { ++numIterations; break; }
        int it = 0;
        st = vcfv_solve(c, so, &it);
        linTotal += it;
        if (st) { status = st; break; }
        kv_sub_update<<<vgrid(c, c->D.NV), kVApi, 0, c->stream>>>(c->D.NV, (const double2*)c->s_x, c->x0);
        if ((st = vcheck(c, "kv_sub_update"))) { status = st; break; }
        ++numIterations;
    }
    if (newtonIts) *newtonIts = numIterations;
    if (linIts) *linIts = linTotal;
    if (errorOut) *errorOut = error;
    if (status) return status;
    if (!converged()) { c->err = "Newton did not converge"; return EWG_ERR_NOT_CONVERGED; }
    return EWG_OK;
}

}  // extern "C"
