// tmx_device.cuh -- geometry, lattice constants and exact FP64 helpers shared
// by the T-mixer kernels.  sm_100a only; compiled with --fmad=false so that no
// multiply-add is contracted implicitly (the reference's x86-64 build has no
// contraction); the only fused operations are the explicit __fma_rn calls of
// div_c() below.
#pragma once
#include <cstdint>

namespace tmx {

// D3Q19 velocity set in the reference's order (Tmixer.cpp:1368-1370).
__host__ __device__ constexpr int EX(int q)
{
    return (q == 1 || q == 7 || q == 10 || q == 11 || q == 14) ? 1
         : (q == 3 || q == 8 || q == 9 || q == 12 || q == 13) ? -1 : 0;
}
__host__ __device__ constexpr int EY(int q)
{
    return (q == 2 || q == 7 || q == 8 || q == 15 || q == 18) ? 1
         : (q == 4 || q == 9 || q == 10 || q == 16 || q == 17) ? -1 : 0;
}
__host__ __device__ constexpr int EZ(int q)
{
    return (q == 5 || q == 11 || q == 12 || q == 15 || q == 16) ? 1
         : (q == 6 || q == 13 || q == 14 || q == 17 || q == 18) ? -1 : 0;
}

// Geometry of one T-mixer: inlet box 0 (inx x iny x nz) and mixing box 1
// (mnx x mny x nz); node g of box b at 1-based (i,j,k) is
// base[b] + ((k-1)*ny[b] + (j-1))*nx[b] + (i-1): x is the contiguous axis, so
// the z and y walls (three quarters of all boundary nodes) are contiguous rows.
// Population q of field f lives at P[(f*19 + q)*ps + g] (structure of arrays,
// ps >= nnodes, a multiple of 64).
struct Geom {
    int inx, iny, nz, mnx, mny, ia, ib;
    int nx[2], ny[2];
    int base[2];
    int nnodes;
    long long ps;
};

// Per-solve physics constants, computed on the host in the reference's order.
struct Phys {
    double c1[4];  // 1.0 - 1.0/tau_f  (flow, A, B, C)
    double c2[4];  // 1.0/tau_f
    double rateconst;
    double rho_out;
    double cin[3][2];
};

__host__ __device__ inline bool is_boundary(const Geom& G, int b, int i, int j, int k)
{
    if (k == 1 || k == G.nz) return true;
    if (b == 0) return i == 1 || i == G.inx || j == G.iny || (j == 1 && (i <= G.ia || i >= G.ib));
    return i == 1 || i == G.mnx || j == 1;
}

// Per-box sizes by selection rather than by indexing: a kernel argument
// indexed with a run-time value would be copied to local memory.
__host__ __device__ inline int box_nx(const Geom& G, int b) { return b ? G.nx[1] : G.nx[0]; }
__host__ __device__ inline int box_ny(const Geom& G, int b) { return b ? G.ny[1] : G.ny[0]; }
__host__ __device__ inline int box_base(const Geom& G, int b) { return b ? G.base[1] : G.base[0]; }

__host__ __device__ inline int node_index(const Geom& G, int b, int i, int j, int k)
{
    return box_base(G, b) + ((k - 1) * box_ny(G, b) + (j - 1)) * box_nx(G, b) + (i - 1);
}

// box and 1-based coordinates of node g
__host__ __device__ inline void decode(const Geom& G, int g, int& b, int& i, int& j, int& k)
{
    b = g >= G.base[1];
    const int l = g - box_base(G, b);
    const int nx = box_nx(G, b), ny = box_ny(G, b);
    i = l % nx + 1;
    const int t = l / nx;
    j = t % ny + 1;
    k = t / ny + 1;
}

// Pull source of direction q for node (b,i,j,k): the reference's streaming()
// (Tmixer.cpp:9039-9347) including the two interface rules (inlet row 1 over
// the opening takes 2,7,8,15,18 from mixing row mny, :9077-9085; mixing row
// mny takes 4,9,10,16,17 from inlet row 1, :9230-9237).  -1 for a source
// outside both boxes (a ghost node; every such value is replaced by a
// boundary closure).
__host__ __device__ inline int pull_src_e(const Geom& G, int b, int i, int j, int k, int ex, int ey, int ez)
{
    int si = i - ex, sj = j - ey, sk = k - ez, sb = b;
    if (b == 0 && j == 1 && ey == 1 && i >= G.ia && i <= G.ib) {
        sb = 1;
        si = i - G.ia + 1 - ex;
        sj = G.mny;
    } else if (b == 1 && j == G.mny && ey == -1) {
        sb = 0;
        si = i + G.ia - 1 - ex;
        sj = 1;
    }
    if (si < 1 || si > box_nx(G, sb) || sj < 1 || sj > box_ny(G, sb) || sk < 1 || sk > G.nz) return -1;
    return node_index(G, sb, si, sj, sk);
}
__host__ __device__ inline int pull_src(const Geom& G, int b, int i, int j, int k, int q)
{
    return pull_src_e(G, b, i, j, k, EX(q), EY(q), EZ(q));
}

// x / d for the constants d = 3, 18, 36, correctly rounded, without a
// division instruction: q0 = RN(x*r) with r = RN(1/d), the exact remainder
// x - d*q0 (one FMA) and one correction FMA.  For these d, r is within
// 2^-54 relative of 1/d, so q0 is within one ulp of x/d and the correction
// returns RN(x/d) (Markstein's theorem; P. Markstein, IBM J. Res. Dev. 34(1),
// 1990).  Valid for x = 0 and for |x| >= 2^-1000 (no subnormal intermediate);
// callers route tinier operands to feq_div_exact().
__device__ __forceinline__ double div_c(double x, double d, double r)
{
    const double q = __dmul_rn(x, r);
    const double e = __fma_rn(-q, d, x);
    return __fma_rn(e, r, q);
}

// q may be a run-time value: the constants are selected, not branched on
__device__ __forceinline__ double feq_div(double x, int q)
{
    const double d = q == 0 ? 3.0 : (q <= 6 ? 18.0 : 36.0);
    const double r = q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0);
    return div_c(x, d, r);
}

__device__ __forceinline__ double feq_div_exact(double x, int q)
{
    return q == 0 ? __ddiv_rn(x, 3.0) : (q <= 6 ? __ddiv_rn(x, 18.0) : __ddiv_rn(x, 36.0));
}

// A density for which rho*poly could fall below 2^-1000 (the equilibrium
// polynomial stays above 1/2 for the lattice velocities a stable run has).
__device__ __forceinline__ bool tiny_density(double r) { return r != 0.0 && fabs(r) < 0x1p-990; }

// lattice weights as the reference stores them (Tmixer.cpp:706-709)
__device__ __forceinline__ double wq(int q) { return q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0); }

// e_q . u as the reference sums it, ((ux*ex + uy*ey) + uz*ez).  The products
// by 0 and +-1 are exact and adding a zero changes at most the sign of a zero
// result (which the equilibrium polynomial absorbs), so only the sum of the
// two non-zero terms rounds; q is a compile-time constant after unrolling.
template <class T>
__device__ __forceinline__ T e_dot_u_e(int ex, int ey, int ez, T ux, T uy, T uz)
{
    const T a = ex > 0 ? ux : -ux, b = ey > 0 ? uy : -uy, c = ez > 0 ? uz : -uz;
    if (ex != 0) return ey != 0 ? a + b : (ez != 0 ? a + c : a);
    if (ey != 0) return ez != 0 ? b + c : b;
    return ez != 0 ? c : T(0);
}
template <class T>
__device__ __forceinline__ T e_dot_u(int q, T ux, T uy, T uz)
{
    return e_dot_u_e(EX(q), EY(q), EZ(q), ux, uy, uz);
}

// Equilibrium polynomial shared by the four fields (they use the flow
// velocity; Tmixer.cpp:1602-1830):
//   q=0:  1.0 - 3.0*u2/2.0
//   q>0:  1.0 + 3.0*eu - 3.0*u2/2.0 + 9.0*eu*eu/2.0   (C left-to-right)
template <class T>
__device__ __forceinline__ void eq_poly(T ux, T uy, T uz, T (&poly)[19])
{
    const T u2 = ux * ux + uy * uy + uz * uz;
    const T t = T(3) * u2 / T(2);
    poly[0] = T(1) - t;
#pragma unroll
    for (int q = 1; q < 19; q++) {
        const T eu = e_dot_u(q, ux, uy, uz);
        poly[q] = T(1) + T(3) * eu - t + T(9) * eu * eu / T(2);
    }
}

// rho = f0 + f1 + ... + f18 in index order (Tmixer.cpp:9391-9560)
template <class T>
__device__ __forceinline__ T sum19(const T (&v)[19])
{
    T s = v[0];
#pragma unroll
    for (int q = 1; q < 19; q++) s += v[q];
    return s;
}

// momentum sums in index order; zero components drop out exactly
// (Tmixer.cpp:9597-9609)
template <class T>
__device__ __forceinline__ void momentum(const T (&f)[19], T& sx, T& sy, T& sz)
{
    sx = f[1] - f[3] + f[7] - f[8] - f[9] + f[10] + f[11] - f[12] - f[13] + f[14];
    sy = f[2] - f[4] + f[7] + f[8] - f[9] - f[10] + f[15] - f[16] - f[17] + f[18];
    sz = f[5] - f[6] + f[11] + f[12] - f[13] - f[14] + f[15] + f[16] - f[17] - f[18];
}

}  // namespace tmx
