// tmx_kernels.cu -- sm_100a kernels of the plain FP64 T-mixer step.
//
// One step of the reference (equilibrium, collision, streaming,
// boundary_conditions, calculate_velocity_density; Tmixer.cpp:10469-10475)
// runs here as two independent launches over disjoint node sets:
//
//   k_bulk      every node that no boundary case touches: pull the 76
//               post-collision populations of the previous step from their
//               upstream neighbours, take moments, equilibrium, BGK collision
//               plus reaction, write the 76 new post-collision populations.
//   k_boundary  every boundary node (compact list, sorted by case): the same,
//               with the reference's closure for its case between the pull
//               and the moments.
//
// The state between steps is the post-collision population set (the
// reference's fn/gn/hn/pn), double-buffered (A-B pull).  Boundary closures
// read, besides their own pulled populations: their own post-collision
// values ("undo streaming"), the previous step's densities of a few nodes
// (kept in R, written by both kernels for the nodes that are read), the
// current step's flow density of an inlet node (recomputed from that node's
// pulled populations), and the pulled species populations of an interior
// node (zero-gradient copies).  None of these is written during the step, so
// all boundary nodes run in parallel and the two kernels need no ordering.
#include <cuda_runtime.h>

#include "tmx_classes.h"
#include "tmx_device.cuh"

namespace tmx {

// ---------------------------------------------------------------------------
// shared per-node physics: equilibrium -> collision -> store
// ---------------------------------------------------------------------------

// Collide one field given its populations f, density r and the shared
// equilibrium polynomial, and store the result.  The reaction source of
// Tmixer.cpp:9697-9761: species A and B (fld 1, 2) lose (w_q*rt)*1.0, C gains
// (w_q*rt)*2.0 (molecular weights Ma = Mb = 1, Mp = 2, :9667).  fld may be a
// run-time value; the arithmetic is the same either way.
__device__ __forceinline__ void collide_store(double* __restrict__ Pout, long long ps, int g, int fld,
                                              const double (&f)[19], double r, const double (&poly)[19],
                                              const Phys& P, double rt)
{
    const double c1 = P.c1[fld], c2 = P.c2[fld];
    double* out = Pout + (long long)fld * 19 * ps + g;
    if (!tiny_density(r)) {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const double feq = feq_div(r * poly[q], q);
            double v = f[q] * c1 + c2 * feq;
            if (fld == 1 || fld == 2) v = v - wq(q) * rt;
            if (fld == 3) v = v + (wq(q) * rt) * 2.0;
            out[(long long)q * ps] = v;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const double feq = feq_div_exact(r * poly[q], q);
            double v = f[q] * c1 + c2 * feq;
            if (fld == 1 || fld == 2) v = v - wq(q) * rt;
            if (fld == 3) v = v + (wq(q) * rt) * 2.0;
            out[(long long)q * ps] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// initial state: f = feq(rho0, 0) for the flow and 0 for the species
// (Tmixer.cpp:1544-1585, 1835-2018), then the first step's collision.
// ---------------------------------------------------------------------------
__global__ void k_init(double* __restrict__ Pout, double* __restrict__ R, double* __restrict__ Mac, Geom G, Phys P,
                       double rho0)
{
    const long long ps = G.ps;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G.nnodes; g += gridDim.x * blockDim.x) {
        double poly[19];
        eq_poly(0.0, 0.0, 0.0, poly);
        double f[19], z[19];
#pragma unroll
        for (int q = 0; q < 19; q++) {
            f[q] = __ddiv_rn(rho0 * poly[q], q == 0 ? 3.0 : (q <= 6 ? 18.0 : 36.0));
            z[q] = __ddiv_rn(0.0 * poly[q], q == 0 ? 3.0 : (q <= 6 ? 18.0 : 36.0));
        }
        const double rt = P.rateconst * 0.0 * 0.0;
        collide_store(Pout, ps, g, 0, f, rho0, poly, P, rt);
        collide_store(Pout, ps, g, 1, z, 0.0, poly, P, rt);
        collide_store(Pout, ps, g, 2, z, 0.0, poly, P, rt);
        collide_store(Pout, ps, g, 3, z, 0.0, poly, P, rt);
        R[g] = rho0;
        R[ps + g] = 0.0;
        R[2 * ps + g] = 0.0;
        R[3 * ps + g] = 0.0;
        Mac[g] = rho0;
#pragma unroll
        for (int m = 1; m < 7; m++) Mac[m * ps + g] = 0.0;
    }
}

// ---------------------------------------------------------------------------
// interior nodes
// ---------------------------------------------------------------------------

// Upstream node of direction q for an interior node: the lattice neighbour in
// the same box, or across the opening for the inlet's row 1 (iface 1: ey = +1
// from mixing row mny) and the mixing box's row mny (iface 2: ey = -1 from
// inlet row 1).  q is a compile-time constant after unrolling.
__device__ __forceinline__ int bulk_src(const Geom& G, int g, int i, int k, int sy, int sz, int iface, int q)
{
    if (EY(q) == 1 && iface == 1) return G.base[1] + ((k - 1 - EZ(q)) * G.mny + (G.mny - 1)) * G.mnx + (i - G.ia - EX(q));
    if (EY(q) == -1 && iface == 2) return ((k - 1 - EZ(q)) * G.iny) * G.inx + (i + G.ia - 2 - EX(q));
    return g - (EX(q) + EY(q) * sy + EZ(q) * sz);
}

__device__ __forceinline__ void bulk_load(const double* __restrict__ Pin, long long ps, int fld, const Geom& G, int g,
                                          int i, int k, int sy, int sz, int iface, double (&v)[19])
{
    const double* base = Pin + (long long)fld * 19 * ps;
#pragma unroll
    for (int q = 0; q < 19; q++) v[q] = __ldg(base + (long long)q * ps + bulk_src(G, g, i, k, sy, sz, iface, q));
}

__global__ void __launch_bounds__(256, 2) k_bulk(const double* __restrict__ Pin, double* __restrict__ Pout,
                                                 double* __restrict__ Rcur, double* __restrict__ Mac, Geom G, Phys P,
                                                 int write_macro)
{
    const long long ps = G.ps;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G.nnodes; g += gridDim.x * blockDim.x) {
        int b, i, j, k;
        decode(G, g, b, i, j, k);
        if (is_boundary(G, b, i, j, k)) continue;
        const int sy = G.nx[b], sz = G.nx[b] * G.ny[b];
        const int iface = (b == 0 && j == 1) ? 1 : ((b == 1 && j == G.mny) ? 2 : 0);

        // flow: moments, equilibrium polynomial (shared by all four fields:
        // they use the flow velocity, Tmixer.cpp:1602-1830), collision
        double poly[19];
        double rho, ux, uy, uz;
        {
            double f[19];
            bulk_load(Pin, ps, 0, G, g, i, k, sy, sz, iface, f);
            rho = sum19(f);
            double sxm, sym, szm;
            momentum(f, sxm, sym, szm);
            ux = sxm / rho;
            uy = sym / rho;
            uz = szm / rho;
            eq_poly(ux, uy, uz, poly);
            collide_store(Pout, ps, g, 0, f, rho, poly, P, 0.0);
        }
        // species A and B: the reaction needs both densities before either
        // collides, so their populations are loaded twice (the second time
        // from cache) rather than held in registers
        double ca, cb;
        {
            double a[19];
            bulk_load(Pin, ps, 1, G, g, i, k, sy, sz, iface, a);
            ca = sum19(a);
            bulk_load(Pin, ps, 2, G, g, i, k, sy, sz, iface, a);
            cb = sum19(a);
        }
        const double rt = P.rateconst * ca * cb;
        double cc;
        {
            double a[19];
            bulk_load(Pin, ps, 1, G, g, i, k, sy, sz, iface, a);
            collide_store(Pout, ps, g, 1, a, ca, poly, P, rt);
            bulk_load(Pin, ps, 2, G, g, i, k, sy, sz, iface, a);
            collide_store(Pout, ps, g, 2, a, cb, poly, P, rt);
            bulk_load(Pin, ps, 3, G, g, i, k, sy, sz, iface, a);
            cc = sum19(a);
            collide_store(Pout, ps, g, 3, a, cc, poly, P, rt);
        }
        // densities the junction edges read next step (Tmixer.cpp:8609, :8851)
        if (b == 0 && j == 2 && (i == G.ia || i == G.ib)) {
            Rcur[g] = rho;
            Rcur[ps + g] = ca;
            Rcur[2 * ps + g] = cb;
            Rcur[3 * ps + g] = cc;
        }
        if (write_macro) {
            Mac[g] = rho;
            Mac[ps + g] = ux;
            Mac[2 * ps + g] = uy;
            Mac[3 * ps + g] = uz;
            Mac[4 * ps + g] = ca;
            Mac[5 * ps + g] = cb;
            Mac[6 * ps + g] = cc;
        }
    }
}

// ---------------------------------------------------------------------------
// boundary closures (Tmixer.cpp:2023-9033)
// ---------------------------------------------------------------------------
struct BCtx {
    const double* __restrict__ Pin;
    const double* __restrict__ Rprev;
    const double* __restrict__ uin1;
    const double* __restrict__ uin2;
    const Geom* G;
    const Phys* P;
    long long ps;
    int g, b, i, j, k;
};

__device__ __forceinline__ double own_fn(const BCtx& c, int fld, int q)
{
    return __ldg(c.Pin + (long long)(fld * 19 + q) * c.ps + c.g);
}
__device__ __forceinline__ double rprev(const BCtx& c, int fld, int b, int i, int j, int k)
{
    return __ldg(c.Rprev + (long long)fld * c.ps + node_index(*c.G, b, i, j, k));
}
__device__ __forceinline__ double uin(const BCtx& c, int side, int j, int k)
{
    return __ldg((side == 0 ? c.uin1 : c.uin2) + j * (c.G->nz + 3) + k);
}
__device__ __forceinline__ void pull_node(const BCtx& c, int fld, int b, int i, int j, int k, double (&v)[19])
{
    const double* base = c.Pin + (long long)fld * 19 * c.ps;
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int s = pull_src(*c.G, b, i, j, k, q);
        v[q] = s >= 0 ? __ldg(base + (long long)q * c.ps + s) : 0.0;
    }
}
// the same sum as sum19 without two directions (the closures' "rho - (...)")
__device__ __forceinline__ double sum_but(const double (&v)[19], int a, int d)
{
    double s = 0.0;
    bool first = true;
#pragma unroll
    for (int q = 0; q < 19; q++) {
        if (q == a || q == d) continue;
        s = first ? v[q] : s + v[q];
        first = false;
    }
    return s;
}
// Zou-He density of the velocity-inlet node (side 0: x=1, side 1: x=inx) as
// the inlet cases compute it this step (Tmixer.cpp:2612-2615, :2675-2678)
__device__ __forceinline__ double inlet_rho_now(const BCtx& c, int side, int j, int k)
{
    double v[19];
    const int x = side == 0 ? 1 : c.G->inx;
    pull_node(c, 0, 0, x, j, k, v);
    const double U = uin(c, side, j, k);
    if (side == 0)
        return (1.0 / (1.0 - U)) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                    2.0 * (v[3] + v[8] + v[9] + v[12] + v[13]));
    return (1.0 / (1.0 + (U))) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                  2.0 * (v[1] + v[7] + v[10] + v[11] + v[14]));
}

// corners: six bounce-backs, buried pairs averaged from their own
// post-collision values, and (corners 1-12) one pair closed from a density.
struct CornerSpec {
    signed char bb[6][2];
    signed char navg;
    signed char avg[3][2];
    signed char cp[2];
};
__constant__ CornerSpec kCorner[16] = {
    {{{1, 3}, {4, 2}, {6, 5}, {10, 8}, {14, 12}, {17, 15}}, 2, {{9, 7}, {11, 13}, {0, 0}}, {16, 18}},    // 1 G'
    {{{3, 1}, {4, 2}, {6, 5}, {17, 15}, {13, 11}, {9, 7}}, 2, {{10, 8}, {12, 14}, {0, 0}}, {16, 18}},    // 2 F'
    {{{1, 3}, {2, 4}, {6, 5}, {7, 9}, {18, 16}, {14, 12}}, 2, {{10, 8}, {11, 13}, {0, 0}}, {15, 17}},    // 3 H'
    {{{3, 1}, {2, 4}, {6, 5}, {8, 10}, {13, 11}, {18, 16}}, 2, {{9, 7}, {12, 14}, {0, 0}}, {15, 17}},    // 4 E'
    {{{1, 3}, {4, 2}, {5, 6}, {16, 18}, {11, 13}, {10, 8}}, 2, {{9, 7}, {14, 12}, {0, 0}}, {15, 17}},    // 5 G
    {{{3, 1}, {4, 2}, {5, 6}, {9, 7}, {12, 14}, {16, 18}}, 2, {{10, 8}, {11, 13}, {0, 0}}, {15, 17}},    // 6 F
    {{{1, 3}, {2, 4}, {5, 6}, {7, 9}, {11, 13}, {15, 17}}, 2, {{10, 8}, {12, 14}, {0, 0}}, {16, 18}},    // 7 H
    {{{3, 1}, {2, 4}, {5, 6}, {8, 10}, {12, 14}, {15, 17}}, 2, {{9, 7}, {11, 13}, {0, 0}}, {16, 18}},    // 8 E
    {{{1, 3}, {2, 4}, {5, 6}, {7, 9}, {11, 13}, {15, 17}}, 2, {{10, 8}, {12, 14}, {0, 0}}, {16, 18}},    // 9 A
    {{{3, 1}, {2, 4}, {5, 6}, {8, 10}, {12, 14}, {15, 17}}, 2, {{9, 7}, {11, 13}, {0, 0}}, {16, 18}},    // 10 B
    {{{1, 3}, {2, 4}, {6, 5}, {7, 9}, {18, 16}, {14, 12}}, 2, {{10, 8}, {11, 13}, {0, 0}}, {15, 17}},    // 11 A'
    {{{3, 1}, {2, 4}, {6, 5}, {8, 10}, {13, 11}, {18, 16}}, 2, {{9, 7}, {12, 14}, {0, 0}}, {15, 17}},    // 12 B'
    {{{6, 5}, {7, 9}, {13, 11}, {14, 12}, {17, 15}, {18, 16}}, 3, {{1, 3}, {4, 2}, {8, 10}}, {-1, -1}},  // 13 D'
    {{{6, 5}, {8, 10}, {13, 11}, {14, 12}, {17, 15}, {18, 16}}, 3, {{9, 7}, {4, 2}, {1, 3}}, {-1, -1}},  // 14 C'
    {{{5, 6}, {8, 10}, {11, 13}, {12, 14}, {15, 17}, {16, 18}}, 3, {{1, 3}, {4, 2}, {9, 7}}, {-1, -1}},  // 15 C
    {{{5, 6}, {7, 9}, {11, 13}, {12, 14}, {15, 17}, {16, 18}}, 3, {{1, 3}, {4, 2}, {8, 10}}, {-1, -1}},  // 16 D
};

// Corner closure on a local copy (runtime indices; 16 nodes per mixer).
__device__ __forceinline__ void corner_closure(const BCtx& c, int fld, int n, double R, double* t)
{
    const CornerSpec& s = kCorner[n];
    for (int m = 0; m < 6; m++) t[s.bb[m][0]] = t[s.bb[m][1]];
    double fa[3];
    for (int m = 0; m < s.navg; m++) fa[m] = (1.0 / 2.0) * (own_fn(c, fld, s.avg[m][0]) + own_fn(c, fld, s.avg[m][1]));
    for (int m = 0; m < s.navg; m++) {
        t[s.avg[m][0]] = fa[m];
        t[s.avg[m][1]] = fa[m];
    }
    if (s.cp[0] >= 0) {
        double sum = 0.0;
        bool first = true;
        for (int q = 0; q < 19; q++) {
            if (q == s.cp[0] || q == s.cp[1]) continue;
            sum = first ? t[q] : sum + t[q];
            first = false;
        }
        t[s.cp[0]] = (1.0 / 2.0) * (R - sum);
        t[s.cp[1]] = t[s.cp[0]];
    }
}

// Apply the closure of class `cls` to field fld of the node in c, on v (the
// node's pulled populations).  Closures follow the reference case by case;
// the comments give the reference lines.  Face classes (inlets, outlet, walls)
// and edge/corner classes are separate functions so that each boundary kernel
// holds only the code of its own classes.
__device__ __forceinline__ void closure_face(const BCtx& c, int cls, int fld, double (&v)[19])
{
    const bool flow = fld == 0;
    switch (cls) {
    case K_INLET1: {  // Inlet1 (:2606-2666)
        if (flow) {
            const double U = uin(c, 0, c.j, c.k);
            const double r = (1.0 / (1.0 - U)) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                                  2.0 * (v[3] + v[8] + v[9] + v[12] + v[13]));
            const double A = (-r * U) / 6.0;
            const double B = (1.0 / 2.0) * (v[2] - v[4] + v[15] - v[16] - v[17] + v[18]);
            const double C = (1.0 / 2.0) * (v[5] - v[6] + v[15] + v[16] - v[17] - v[18]);
            v[1] = v[3] + (r * U) / 3.0;
            v[7] = v[9] - (A + B); v[10] = v[8] - (A - B); v[11] = v[13] - (A + C); v[14] = v[12] - (A - C);
        } else {
            const double cin = c.P->cin[fld - 1][0];
            v[1] = -v[3] + (2.0 / 18.0) * cin;
            v[7] = -v[9] + (2.0 / 36.0) * cin;
            v[10] = -v[8] + (2.0 / 36.0) * cin;
            v[11] = -v[13] + (2.0 / 36.0) * cin;
            v[14] = -v[12] + (2.0 / 36.0) * cin;
        }
    } break;
    case K_INLET2: {  // Inlet2 (:2668-2730)
        if (flow) {
            const double U = uin(c, 1, c.j, c.k);
            const double r = (1.0 / (1.0 + (U))) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                                    2.0 * (v[1] + v[7] + v[10] + v[11] + v[14]));
            const double A = (-r * (U)) / 6.0;
            const double B = (1.0 / 2.0) * (v[2] - v[4] + v[15] - v[16] - v[17] + v[18]);
            const double C = (1.0 / 2.0) * (v[5] - v[6] + v[15] + v[16] - v[17] - v[18]);
            v[3] = v[1] - (r * (U)) / 3.0;
            v[9] = v[7] + (A + B); v[8] = v[10] + (A - B); v[13] = v[11] + (A + C); v[12] = v[14] + (A - C);
        } else {
            const double cin = c.P->cin[fld - 1][1];
            v[3] = -v[1] + (2.0 / 18.0) * cin;
            v[9] = -v[7] + (2.0 / 36.0) * cin;
            v[8] = -v[10] + (2.0 / 36.0) * cin;
            v[13] = -v[11] + (2.0 / 36.0) * cin;
            v[12] = -v[14] + (2.0 / 36.0) * cin;
        }
    } break;
    case K_FACE_YT: {  // Case 10 flow (:2731-2764); species copy from y-1 (:2766-2872)
        if (flow) {
            const double C = (1.0 / 2.0) * (v[5] - v[6] + v[11] + v[12] - v[13] - v[14]);
            v[4] = v[2]; v[16] = v[18] - C; v[17] = v[15] + C;
            const double A = (1.0 / 2.0) * (v[1] - v[3] + v[11] - v[12] - v[13] + v[14]);
            v[9] = v[7] + A; v[10] = v[8] - A;
        } else pull_node(c, fld, c.b, c.i, c.j - 1, c.k, v);
    } break;
    case K_FACE_Y1: {  // Cases 11, 12 flow (:2874-2906, :3016-3049); species copy from y+1
        if (flow) {
            const double C = (1.0 / 2.0) * (v[5] - v[6] + v[11] + v[12] - v[13] - v[14]);
            v[2] = v[4]; v[15] = v[17] - C; v[18] = v[16] + C;
            const double A = (1.0 / 2.0) * (v[1] - v[3] + v[11] - v[12] - v[13] + v[14]);
            v[7] = v[9] - A; v[8] = v[10] + A;
        } else pull_node(c, fld, c.b, c.i, c.j + 1, c.k, v);
    } break;
    case K_OUTLET: {  // Case 13 flow (:3162-3190); species copy from y+1 (:3192-3273)
        if (flow) {
            const double rout = c.P->rho_out;
            const double uy = 1.0 - (1.0 / rout) * ((v[0] + v[1] + v[3] + v[5] + v[6] + v[11] + v[12] + v[13] + v[14]) +
                                                    2.0 * (v[4] + v[9] + v[10] + v[16] + v[17]));
            const double A = (rout * uy) / 6.0;
            const double B = (1.0 / 2.0) * ((v[3] + v[12] + v[13]) - (v[1] + v[11] + v[14]));
            const double C = (1.0 / 2.0) * ((v[6] + v[13] + v[14]) - (v[5] + v[11] + v[12]));
            v[2] = v[4] + (rout * uy) / 3.0;
            v[7] = v[9] + (A + B); v[8] = v[10] + (A - B); v[15] = v[17] + (A + C); v[18] = v[16] + (A - C);
        } else pull_node(c, fld, c.b, c.i, c.j + 1, c.k, v);
    } break;
    case K_FACE_MX1: {  // Case 14 (:3275-3404)
        if (flow) {
            const double C = (1.0 / 2.0) * ((v[6] + v[17] + v[18]) - (v[5] + v[15] + v[16]));
            v[1] = v[3]; v[11] = v[13] + (C); v[14] = v[12] - (C);
            const double A = (1.0 / 2.0) * ((v[2] + v[15] + v[18]) - (v[4] + v[16] + v[17]));
            v[7] = v[9] - A; v[10] = v[8] + A;
        } else pull_node(c, fld, c.b, c.i + 1, c.j, c.k, v);
    } break;
    case K_FACE_MXT: {  // Case 15 (:3405-3539)
        if (flow) {
            const double C = (1.0 / 2.0) * ((v[6] + v[17] + v[18]) - (v[5] + v[15] + v[16]));
            v[3] = v[1]; v[13] = v[11] - (C); v[12] = v[14] + (C);
            const double A = (1.0 / 2.0) * ((v[2] + v[15] + v[18]) - (v[4] + v[16] + v[17]));
            v[9] = v[7] + A; v[8] = v[10] - A;
        } else pull_node(c, fld, c.b, c.i - 1, c.j, c.k, v);
    } break;
    case K_FACE_ZT: {  // Cases 16, 17 and the opening nodes of 17 (:3540-3887)
        if (flow) {
            const double B = (1.0 / 2.0) * (v[2] - v[4] + v[7] + v[8] - v[9] - v[10]);
            v[6] = v[5]; v[17] = v[15] + B; v[18] = v[16] - B;
            const double A = (1.0 / 2.0) * (v[1] - v[3] + v[7] - v[8] - v[9] + v[10]);
            v[13] = v[11] + A; v[14] = v[12] - A;
        } else pull_node(c, fld, c.b, c.i, c.j, c.k - 1, v);
    } break;
    case K_FACE_Z1: {  // Cases 18, 19 and the opening nodes of 19 (:3888-4237)
        if (flow) {
            const double B = (1.0 / 2.0) * (v[2] - v[4] + v[7] + v[8] - v[9] - v[10]);
            v[5] = v[6]; v[15] = v[17] - B; v[16] = v[18] + B;
            const double A = (1.0 / 2.0) * (v[1] - v[3] + v[7] - v[8] - v[9] + v[10]);
            v[11] = v[13] - A; v[12] = v[14] + A;
        } else pull_node(c, fld, c.b, c.i, c.j, c.k + 1, v);
    } break;
    default: break;
    }
}

__device__ __forceinline__ void closure_edge(const BCtx& c, int cls, int fld, double (&v)[19])
{
    const Geom& G = *c.G;
    const bool flow = fld == 0;
    switch (cls) {
    case K_EDGE_Y1_ZTOP: {  // Cases 2, 3 (:2030-2342)
        v[2] = v[4]; v[6] = v[5]; v[7] = v[9]; v[8] = v[10]; v[13] = v[11]; v[14] = v[12]; v[18] = v[16];
        v[15] = (1.0 / 2.0) * (own_fn(c, fld, 15) + own_fn(c, fld, 17));
        v[17] = v[15];
        const double A = (1.0 / 4.0) * (v[1] - v[3]);
        v[7] = v[9] - A; v[8] = v[10] + A; v[13] = v[11] + A; v[14] = v[12] - A;
    } break;
    case K_EDGE_X1_ZTOP: {  // Case 4 (:2343-2476); field C keeps p13 = pn13 (:2474)
        const double B = 1.0 / 4.0 * (v[2] - v[4]);
        v[1] = v[3]; v[6] = v[5]; v[7] = v[9] - B; v[10] = v[8] + B; v[14] = v[12]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[13] = own_fn(c, fld, 13);
        v[11] = (1.0 / 2.0) * (rprev(c, fld, 0, 1, c.j, G.nz - 1) - sum_but(v, 11, 13));
        if (fld != 3) v[13] = v[11];
    } break;
    case K_EDGE_XT_ZTOP: {  // Case 6 (:2477-2605)
        const double B = (1.0 / 4.0) * (v[2] - v[4]);
        v[3] = v[1]; v[6] = v[5]; v[9] = v[7] + B; v[8] = v[10] - B; v[13] = v[11]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[12] = (1.0 / 2.0) * (rprev(c, fld, 0, G.inx, c.j, G.nz - 1) - sum_but(v, 12, 14));
        v[14] = v[12];
    } break;
    case K_EDGE_YT_ZT: {  // Case 20 (:4238-4385)
        v[4] = v[2]; v[6] = v[5]; v[17] = v[15];
        v[16] = (1.0 / 2.0) * (own_fn(c, fld, 16) + own_fn(c, fld, 18));
        v[18] = v[16];
        const double A = (1.0 / 4.0) * (v[1] - v[3]);
        v[9] = v[7] + A; v[10] = v[8] - A; v[13] = v[11] + A; v[14] = v[12] - A;
    } break;
    case K_EDGE_YT_Z1: {  // Case 21 (:4386-4533)
        v[4] = v[2]; v[5] = v[6]; v[16] = v[18];
        v[15] = (1.0 / 2.0) * (own_fn(c, fld, 15) + own_fn(c, fld, 17));
        v[17] = v[15];
        const double A = (1.0 / 4.0) * (v[1] - v[3]);
        v[9] = v[7] + A; v[10] = v[8] - A; v[11] = v[13] - A; v[12] = v[14] + A;
    } break;
    case K_EDGE_X1_Z1: {  // Case 22 (:4534-4656); flow density of (1,j,2) from this step
        const double B = 1.0 / 4.0 * (v[2] - v[4]);
        v[1] = v[3]; v[5] = v[6]; v[7] = v[9] - B; v[10] = v[8] + B; v[11] = v[13]; v[15] = v[17] - B; v[16] = v[18] + B;
        const double R = flow ? inlet_rho_now(c, 0, c.j, 2) : rprev(c, fld, 0, 1, c.j, 2);
        v[12] = (1.0 / 2.0) * (R - sum_but(v, 12, 14));
        v[14] = v[12];
    } break;
    case K_EDGE_XT_Z1: {  // Case 23 (:4657-4779)
        const double B = 1.0 / 4.0 * (v[2] - v[4]);
        v[3] = v[1]; v[5] = v[6]; v[8] = v[10] - B; v[9] = v[7] + B; v[12] = v[14]; v[15] = v[17] - B; v[16] = v[18] + B;
        const double R = flow ? inlet_rho_now(c, 1, c.j, 2) : rprev(c, fld, 0, G.inx, c.j, 2);
        v[11] = (1.0 / 2.0) * (R - sum_but(v, 11, 13));
        v[13] = v[11];
    } break;
    case K_EDGE_X1_Y1: {  // Case 24 (:4780-4909)
        const double C = 1.0 / 4.0 * (v[5] - v[6]);
        v[1] = v[3]; v[2] = v[4]; v[7] = v[9]; v[11] = v[13] - C; v[14] = v[12] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const double R = flow ? inlet_rho_now(c, 0, 2, c.k) : rprev(c, fld, 0, 1, 2, c.k);
        v[8] = (1.0 / 2.0) * (R - sum_but(v, 8, 10));
        v[10] = v[8];
    } break;
    case K_EDGE_X1_YT: {  // Case 25 (:4910-5032)
        const double C = 1.0 / 4.0 * (v[5] - v[6]);
        v[1] = v[3]; v[4] = v[2]; v[10] = v[8]; v[11] = v[13] - C; v[14] = v[12] + C; v[16] = v[18] - C; v[17] = v[15] + C;
        const double R = flow ? inlet_rho_now(c, 0, G.iny - 1, c.k) : rprev(c, fld, 0, 1, G.iny - 1, c.k);
        v[7] = (1.0 / 2.0) * (R - sum_but(v, 7, 9));
        v[9] = v[7];
    } break;
    case K_EDGE_XT_Y1: {  // Case 26 (:5033-5159)
        const double C = 1.0 / 4.0 * (v[5] - v[6]);
        v[3] = v[1]; v[2] = v[4]; v[8] = v[10]; v[12] = v[14] - C; v[13] = v[11] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const double R = flow ? inlet_rho_now(c, 1, 2, c.k) : rprev(c, fld, 0, G.inx, 2, c.k);
        v[7] = (1.0 / 2.0) * (R - sum_but(v, 7, 9));
        v[9] = v[7];
    } break;
    case K_EDGE_XT_YT: {  // Case 27 (:5160-5281)
        const double C = 1.0 / 4.0 * (v[5] - v[6]);
        v[3] = v[1]; v[4] = v[2]; v[9] = v[7]; v[12] = v[14] - C; v[13] = v[11] + C; v[16] = v[18] - C; v[17] = v[15] + C;
        const double R = flow ? inlet_rho_now(c, 1, G.iny - 1, c.k) : rprev(c, fld, 0, G.inx, G.iny - 1, c.k);
        v[8] = (1.0 / 2.0) * (R - sum_but(v, 8, 10));
        v[10] = v[8];
    } break;
    case K_EDGE_Y1_Z1: {  // Cases 28, 29 (:5282-5571)
        v[2] = v[4]; v[5] = v[6]; v[15] = v[17];
        v[16] = (1.0 / 2.0) * (own_fn(c, fld, 16) + own_fn(c, fld, 18));
        v[18] = v[16];
        const double A = (1.0 / 4.0) * (v[1] - v[3]);
        v[7] = v[9] - A; v[8] = v[10] + A; v[11] = v[13] - A; v[12] = v[14] + A;
    } break;
    case K_MEDGE_AB: {  // (:7788-7868)
        const double A = (1.0 / 4.0) * (v[1] - v[3]);
        v[2] = v[4]; v[5] = v[6]; v[7] = v[9] - A; v[8] = v[10] + A; v[11] = v[13] - A; v[12] = v[14] + A; v[15] = v[17];
        const double R = flow ? c.P->rho_out : rprev(c, fld, 1, c.i, 2, 1);
        v[18] = (1.0 / 2.0) * (R - sum_but(v, 16, 18));
        v[16] = v[18];
    } break;
    case K_MEDGE_ApBp: {  // (:7870-7950)
        const double A = (1.0 / 4.0) * (v[1] - v[3]);
        v[2] = v[4]; v[6] = v[5]; v[7] = v[9] - A; v[8] = v[10] + A; v[13] = v[11] + A; v[14] = v[12] - A; v[18] = v[16];
        const double R = flow ? c.P->rho_out : rprev(c, fld, 1, c.i, 2, G.nz);
        v[15] = (1.0 / 2.0) * (R - sum_but(v, 15, 17));
        v[17] = v[15];
    } break;
    case K_MEDGE_AAp: {  // (:7951-8043)
        const double C = (1.0 / 4.0) * (v[5] - v[6]);
        v[1] = v[3]; v[2] = v[4]; v[7] = v[9]; v[11] = v[13] - C; v[14] = v[12] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const double R = flow ? c.P->rho_out : rprev(c, fld, 1, 1, 2, c.k);
        v[8] = (1.0 / 2.0) * (R - sum_but(v, 8, 10));
        v[10] = v[8];
    } break;
    case K_MEDGE_BBp: {  // (:8044-8136)
        const double C = (1.0 / 4.0) * (v[5] - v[6]);
        v[3] = v[1]; v[2] = v[4]; v[8] = v[10]; v[12] = v[14] - C; v[13] = v[11] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const double R = flow ? c.P->rho_out : rprev(c, fld, 1, G.mnx, 2, c.k);
        v[7] = (1.0 / 2.0) * (R - sum_but(v, 7, 9));
        v[9] = v[7];
    } break;
    case K_MEDGE_AD: {  // (:8137-8244)
        const double B = (1.0 / 4.0) * (v[2] - v[4]);
        v[1] = v[3]; v[5] = v[6]; v[7] = v[9] - B; v[10] = v[8] + B; v[11] = v[13]; v[15] = v[17] - B; v[16] = v[18] + B;
        v[14] = (1.0 / 2.0) * (own_fn(c, fld, 12) + own_fn(c, fld, 14));
        v[12] = v[14];
    } break;
    case K_MEDGE_ApDp: {  // (:8245-8344)
        const double B = (1.0 / 4.0) * (v[2] - v[4]);
        v[1] = v[3]; v[6] = v[5]; v[7] = v[9] - B; v[10] = v[8] + B; v[14] = v[12]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[13] = (1.0 / 2.0) * (own_fn(c, fld, 11) + own_fn(c, fld, 13));
        v[11] = v[13];
    } break;
    case K_MEDGE_BC: {  // (:8345-8445)
        const double B = (1.0 / 4.0) * (v[2] - v[4]);
        v[3] = v[1]; v[5] = v[6]; v[8] = v[10] - B; v[9] = v[7] + B; v[12] = v[14]; v[15] = v[17] - B; v[16] = v[18] + B;
        v[13] = (1.0 / 2.0) * (own_fn(c, fld, 11) + own_fn(c, fld, 13));
        v[11] = v[13];
    } break;
    case K_MEDGE_BpCp: {  // (:8446-8550)
        const double B = (1.0 / 4.0) * (v[2] - v[4]);
        v[3] = v[1]; v[6] = v[5]; v[9] = v[7] + B; v[8] = v[10] - B; v[13] = v[11]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[14] = (1.0 / 2.0) * (own_fn(c, fld, 12) + own_fn(c, fld, 14));
        v[12] = v[14];
    } break;
    case K_JUNC_DD:    // (:8551-8792): closed pair 7/9 from the density at (ia, 2, k)
    case K_JUNC_CC: {  // (:8793-9033): closed pair 8/10 from the density at (ib, 2, k)
        const bool dd = cls == K_JUNC_DD;
        double a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 3) + own_fn(c, fld, 1)); v[3] = a; v[1] = a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 4) + own_fn(c, fld, 2)); v[4] = a; v[2] = a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 5) + own_fn(c, fld, 6)); v[6] = a; v[5] = a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 11) + own_fn(c, fld, 13)); v[13] = a; v[11] = a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 12) + own_fn(c, fld, 14)); v[14] = a; v[12] = a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 15) + own_fn(c, fld, 17)); v[17] = a; v[15] = a;
        a = (1.0 / 2.0) * (own_fn(c, fld, 16) + own_fn(c, fld, 18)); v[18] = a; v[16] = a;
        const double R = rprev(c, fld, 0, dd ? G.ia : G.ib, 2, c.k);
        if (dd) {
            a = (1.0 / 2.0) * (own_fn(c, fld, 8) + own_fn(c, fld, 10)); v[10] = a; v[8] = a;
            v[7] = (1.0 / 2.0) * (R - sum_but(v, 7, 9));
            v[9] = v[7];
        } else {
            a = (1.0 / 2.0) * (own_fn(c, fld, 7) + own_fn(c, fld, 9)); v[9] = a; v[7] = a;
            v[8] = (1.0 / 2.0) * (R - sum_but(v, 8, 10));
            v[10] = v[8];
        }
    } break;
    default: {
        if (cls >= K_CORNER_1 && cls <= K_CORNER_16) {
            const int n = cls - K_CORNER_1;
            double R = 0.0;
            if (n < 8) {  // inlet corners: density of the adjacent x-y edge node
                R = rprev(c, fld, 0, c.i, c.j, c.k == G.nz ? G.nz - 1 : 2);
            } else if (n < 12) {  // outlet corners: rho_out; species read the row
                R = flow ? c.P->rho_out : 0.0;  // below the outlet, which is 0
            }
            double t[19];
#pragma unroll
            for (int q = 0; q < 19; q++) t[q] = v[q];
            corner_closure(c, fld, n, R, t);
#pragma unroll
            for (int q = 0; q < 19; q++) v[q] = t[q];
        }
    } break;
    }
}

// The post-closure populations of field fld of the boundary node in c.  A
// species on a wall face is a zero-gradient copy of an interior node's pulled
// populations (Tmixer.cpp:2766-4237), so it pulls that node directly.
template <bool FACES>
__device__ __forceinline__ void closed_pull(const BCtx& c, int cls, int fld, double (&v)[19])
{
    if (FACES && fld > 0) {
        int di = 0, dj = 0, dk = 0;
        switch (cls) {
        case K_FACE_YT: dj = -1; break;
        case K_FACE_Y1:
        case K_OUTLET: dj = 1; break;
        case K_FACE_MX1: di = 1; break;
        case K_FACE_MXT: di = -1; break;
        case K_FACE_ZT: dk = -1; break;
        case K_FACE_Z1: dk = 1; break;
        default: break;
        }
        if (di | dj | dk) {
            pull_node(c, fld, c.b, c.i + di, c.j + dj, c.k + dk, v);
            return;
        }
    }
    pull_node(c, fld, c.b, c.i, c.j, c.k, v);
    if (FACES)
        closure_face(c, cls, fld, v);
    else
        closure_edge(c, cls, fld, v);
}

// ---------------------------------------------------------------------------
// boundary nodes: one thread per node of a compact, class-sorted list; FACES
// selects the list of inlet/outlet/wall-face nodes or of edge/corner nodes.
// The closed species A and B populations wait in shared memory while the
// reaction term (which needs both densities) is formed.
// ---------------------------------------------------------------------------
constexpr int kBoundaryThreads = 128;

template <bool FACES>
__device__ __forceinline__ void boundary_body(const double* __restrict__ Pin, double* __restrict__ Pout,
                                              const double* __restrict__ Rprev, double* __restrict__ Rcur,
                                              double* __restrict__ Mac, const int* __restrict__ bnode,
                                              const unsigned char* __restrict__ bcls, int nb,
                                              const double* __restrict__ uin1, const double* __restrict__ uin2,
                                              const Geom& G, const Phys& P, int write_macro)
{
    __shared__ double stash[2][19][kBoundaryThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    BCtx c;
    c.Pin = Pin;
    c.Rprev = Rprev;
    c.uin1 = uin1;
    c.uin2 = uin2;
    c.G = &G;
    c.P = &P;
    c.ps = G.ps;
    c.g = bnode[t];
    decode(G, c.g, c.b, c.i, c.j, c.k);
    const int cls = bcls[t];
    const long long ps = G.ps;
    const bool outlet = c.b == 1 && c.j == 1;
    const int tx = threadIdx.x;

    double poly[19];
    double rho, ux, uy, uz;
    {
        double f[19];
        closed_pull<FACES>(c, cls, 0, f);
        // the outlet row's density is pinned to rho_out (Tmixer.cpp:9575-9582)
        rho = outlet ? P.rho_out : sum19(f);
        double sxm, sym, szm;
        momentum(f, sxm, sym, szm);
        ux = sxm / rho;
        uy = sym / rho;
        uz = szm / rho;
        eq_poly(ux, uy, uz, poly);
        collide_store(Pout, ps, c.g, 0, f, rho, poly, P, 0.0);
    }
    double ca, cb, cc;
    {
        double v[19];
        closed_pull<FACES>(c, cls, 1, v);
        ca = sum19(v);
#pragma unroll
        for (int q = 0; q < 19; q++) stash[0][q][tx] = v[q];
        closed_pull<FACES>(c, cls, 2, v);
        cb = sum19(v);
#pragma unroll
        for (int q = 0; q < 19; q++) stash[1][q][tx] = v[q];
    }
    const double rt = P.rateconst * ca * cb;
    {
        double v[19];
#pragma unroll
        for (int q = 0; q < 19; q++) v[q] = stash[0][q][tx];
        collide_store(Pout, ps, c.g, 1, v, ca, poly, P, rt);
#pragma unroll
        for (int q = 0; q < 19; q++) v[q] = stash[1][q][tx];
        collide_store(Pout, ps, c.g, 2, v, cb, poly, P, rt);
        closed_pull<FACES>(c, cls, 3, v);
        cc = sum19(v);
        collide_store(Pout, ps, c.g, 3, v, cc, poly, P, rt);
    }

    Rcur[c.g] = rho;
    Rcur[ps + c.g] = ca;
    Rcur[2 * ps + c.g] = cb;
    Rcur[3 * ps + c.g] = cc;
    if (write_macro) {
        Mac[c.g] = rho;
        Mac[ps + c.g] = ux;
        Mac[2 * ps + c.g] = uy;
        Mac[3 * ps + c.g] = uz;
        Mac[4 * ps + c.g] = ca;
        Mac[5 * ps + c.g] = cb;
        Mac[6 * ps + c.g] = cc;
    }
}

__global__ void __launch_bounds__(kBoundaryThreads)
    k_boundary_faces(const double* __restrict__ Pin, double* __restrict__ Pout, const double* __restrict__ Rprev,
                     double* __restrict__ Rcur, double* __restrict__ Mac, const int* __restrict__ bnode,
                     const unsigned char* __restrict__ bcls, int nb, const double* __restrict__ uin1,
                     const double* __restrict__ uin2, Geom G, Phys P, int write_macro)
{
    boundary_body<true>(Pin, Pout, Rprev, Rcur, Mac, bnode, bcls, nb, uin1, uin2, G, P, write_macro);
}

__global__ void __launch_bounds__(kBoundaryThreads)
    k_boundary_edges(const double* __restrict__ Pin, double* __restrict__ Pout, const double* __restrict__ Rprev,
                     double* __restrict__ Rcur, double* __restrict__ Mac, const int* __restrict__ bnode,
                     const unsigned char* __restrict__ bcls, int nb, const double* __restrict__ uin1,
                     const double* __restrict__ uin2, Geom G, Phys P, int write_macro)
{
    boundary_body<false>(Pin, Pout, Rprev, Rcur, Mac, bnode, bcls, nb, uin1, uin2, G, P, write_macro);
}

// ---------------------------------------------------------------------------
// mixing quality (Tmixer.cpp:10161-10409): per row, per species, the sums of
// the reference in its order (k inner, i outer), then per-row maxima.  One
// thread block per row; thread s handles species s.  Rows: mixing 1..mny,
// then inlet 1..iny over x = ia..ib.
// ---------------------------------------------------------------------------
__global__ void k_mixing_rows(const double* __restrict__ Mac, Geom G, double* __restrict__ stats)
{
    const int row = blockIdx.x;
    const int s = threadIdx.x;
    if (s >= 3) return;
    const int b = row < G.mny ? 1 : 0;
    const int j = b == 1 ? row + 1 : row - G.mny + 1;
    const int i0 = b == 1 ? 1 : G.ia, i1 = b == 1 ? G.mnx : G.ib;
    const double* cfield = Mac + (long long)(4 + s) * G.ps;
    double sumx = 0.0, mx = __longlong_as_double(0xfff0000000000000ULL);  // -inf
    for (int i = i0; i <= i1; i++) {
        double sumz = 0.0;
        for (int k = 1; k <= G.nz; k++) {
            const double v = cfield[node_index(G, b, i, j, k)];
            sumz += v;
            mx = fmax(mx, v);
        }
        sumx += sumz;
    }
    const double avg = (sumx / (1.0 * G.nz * G.mnx));
    sumx = 0.0;
    for (int i = i0; i <= i1; i++) {
        double sumz = 0.0;
        for (int k = 1; k <= G.nz; k++) {
            const double d = cfield[node_index(G, b, i, j, k)] - avg;
            sumz += d * d;
        }
        sumx += sumz;
    }
    const double var = (1.0 / (1.0 * G.nz * G.mnx)) * sumx;
    stats[row * 9 + s] = avg;
    stats[row * 9 + 3 + s] = var;
    stats[row * 9 + 6 + s] = mx;
}

// ---------------------------------------------------------------------------
// FP64 totals: warp-shuffle block reduction, one partial per block
// ---------------------------------------------------------------------------
__global__ void k_sums(const double* __restrict__ Mac, Geom G, double* __restrict__ partial)
{
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G.nnodes; g += gridDim.x * blockDim.x) {
        const double r = Mac[g], a = Mac[4 * G.ps + g], b2 = Mac[5 * G.ps + g], c3 = Mac[6 * G.ps + g];
        acc[0] += r;
        acc[1] += a;
        acc[2] += b2;
        acc[3] += c3;
        int b, i, j, k;
        decode(G, g, b, i, j, k);
        if (b == 1 && j == 1) acc[4] += r * Mac[2 * G.ps + g];
        const double uxv = Mac[G.ps + g], uyv = Mac[2 * G.ps + g], uzv = Mac[3 * G.ps + g];
        if (!isfinite(r) || !isfinite(a) || !isfinite(b2) || !isfinite(c3) || !isfinite(uxv) || !isfinite(uyv) ||
            !isfinite(uzv))
            acc[5] += 1.0;
    }
    __shared__ double sh[6][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < 6; m++) {
        double v = acc[m];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[m][w] = v;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int m = 0; m < 6; m++) {
            double v = lane < nw ? sh[m][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) partial[blockIdx.x * 6 + m] = v;
        }
    }
}

}  // namespace tmx
