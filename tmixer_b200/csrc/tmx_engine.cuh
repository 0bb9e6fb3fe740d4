// tmx_engine.cuh -- the T-mixer step as device code templated on a precision
// policy PR (scalar type T of the arithmetic, storage type S of the
// populations).  The kernels that instantiate it live in tmx_kernels.cu (FP64,
// compiled without contraction: bit-exact with the reference) and
// tmx_kernels_lp.cu (FP32 arithmetic; FP32 storage, or FP16 storage of the
// non-equilibrium part next to FP32 moment records).
//
// One step of the reference (equilibrium, collision, streaming,
// boundary_conditions, calculate_velocity_density; Tmixer.cpp:10469-10475)
// runs as launches over disjoint node sets:
//
//   bulk      every node that no boundary case touches: pull the 76
//             post-collision populations of the previous step from their
//             upstream neighbours, take moments, equilibrium, BGK collision
//             plus reaction, write the 76 new post-collision populations.
//   boundary  every boundary node (compact list, sorted by case; faces and
//             edges/corners in two kernels): the same, with the reference's
//             closure for its case between the pull and the moments.
//
// The state between steps is the post-collision population set (the
// reference's fn/gn/hn/pn), double-buffered (A-B pull).  Boundary closures
// read, besides their own pulled populations: their own post-collision
// values ("undo streaming"), the previous step's densities of a few nodes
// (kept in R, written by both kernels for the nodes that are read), the
// current step's flow density of an inlet node (recomputed from that node's
// pulled populations), and the pulled species populations of an interior
// node (zero-gradient copies).  None of these is written during the step, so
// all boundary nodes run in parallel and the kernels need no ordering.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tmx_classes.h"
#include "tmx_device.cuh"
#include "tmx_kernels.cuh"

namespace tmx {

// ---------------------------------------------------------------------------
// precision policies
// ---------------------------------------------------------------------------

// FP32 equilibrium polynomial of the reduced-precision forms, evaluated the
// same way by every caller: P_q = omt + e.u (3 + 4.5 e.u) as two correctly
// rounded fused multiply-adds, with omt = 1 - 1.5 |u|^2 shared by the 19
// directions.  The FP16 form adds and subtracts w_q * rho * P_q when it
// encodes and decodes populations, so writer and reader must produce the same
// bits from the same inputs: explicit __fmaf_rn / __fmul_rn / __fadd_rn, never
// left to contraction.  The FP16 form stores omt with the writer's moments so
// that readers need not recompute it.
__device__ __forceinline__ float omt_term(float ux, float uy, float uz)
{
    const float u2 = __fadd_rn(__fadd_rn(__fmul_rn(ux, ux), __fmul_rn(uy, uy)), __fmul_rn(uz, uz));
    return __fsub_rn(1.0f, __fmul_rn(1.5f, u2));
}
// direction given by its lattice vector (ex, ey, ez), possibly run-time values
__device__ __forceinline__ float poly_e_omt(int ex, int ey, int ez, float ux, float uy, float uz, float omt)
{
    if ((ex | ey | ez) == 0) return omt;
    const float eu = e_dot_u_e(ex, ey, ez, ux, uy, uz);
    return __fmaf_rn(eu, __fmaf_rn(4.5f, eu, 3.0f), omt);
}
__device__ __forceinline__ float poly_q_omt(int q, float ux, float uy, float uz, float omt)
{
    return poly_e_omt(EX(q), EY(q), EZ(q), ux, uy, uz, omt);
}

// Collision of one direction of the FP32 form with sm_100's packed
// two-wide FP32 arithmetic, on the field pairs (flow, A) and (B, C): given
// the pulled values, the densities, w_q * poly_q (pw) and w_q * rate (wrt),
// the equilibria f = r * pw and the post-collision values
// o = in + c2 * (f - in), A and B minus wrt, C plus 2 wrt.  (The same value
// as in * c1 + c2 * f with c1 = 1 - c2, but rounding one small difference:
// with c2 = 1/tau near 2, as for tau_c = 0.55, the two large terms of
// opposite sign cost the species fields several times the FP32 rounding per
// step.)  c1 is not used.  (The FP16-storage form stores o - f, which
// F16::collide_store forms directly.)
__device__ __forceinline__ void collide_pairs(float2 in01, float2 in23, float2 r01, float2 r23, float pw, float2,
                                              float2, float2 c2a, float2 c2b, float wrt, float2& o01, float2& o23,
                                              float2& f01, float2& f23)
{
    const float2 pp = make_float2(pw, pw);
    f01 = __fmul2_rn(r01, pp);
    f23 = __fmul2_rn(r23, pp);
    o01 = __ffma2_rn(c2a, __fadd2_rn(f01, make_float2(-in01.x, -in01.y)), in01);
    o23 = __ffma2_rn(c2b, __fadd2_rn(f23, make_float2(-in23.x, -in23.y)), in23);
    o01 = __fadd2_rn(o01, make_float2(0.0f, -wrt));
    o23 = __fadd2_rn(o23, make_float2(-wrt, 2.0f * wrt));
}

// Plain form: FP64 storage and arithmetic, operation by operation as the
// reference (the translation unit is compiled with --fmad=false); the
// equilibrium divisions are correctly rounded (div_c).
struct F64 {
    using T = double;
    using S = double;
    static constexpr bool kMoments = false;
    static constexpr bool kOnePass = false;  // 76 FP64 values exceed the register budget
    // structure of arrays: plane (fld, q) of ps values, nodes x-fastest
    __host__ __device__ static long long off(int fld, int q, long long ps, long long g)
    {
        return (long long)(fld * 19 + q) * ps + g;
    }
    __device__ static void poly(T ux, T uy, T uz, T (&p)[19]) { eq_poly(ux, uy, uz, p); }
    __device__ static bool tiny(T r) { return tiny_density(r); }
    __device__ static T feq(T r, T polyq, int q, bool tiny)
    {
        const T x = r * polyq;
        return tiny ? feq_div_exact(x, q) : feq_div(x, q);
    }
    __device__ static T decode(const S* p, int, int, const float4*, long long, int) { return __ldg(p); }
    __device__ static void encode(S* p, T v, T) { *p = v; }
    // the equilibrium polynomial of one direction given by (ex, ey, ez), with
    // the operations of eq_poly (the weight enters through feq's division)
    __device__ static T pw_dir(int ex, int ey, int ez, T, T ux, T uy, T uz)
    {
        const T u2 = ux * ux + uy * uy + uz * uz;
        const T t = T(3) * u2 / T(2);
        if ((ex | ey | ez) == 0) return T(1) - t;
        const T eu = e_dot_u_e(ex, ey, ez, ux, uy, uz);
        return T(1) + T(3) * eu - t + T(9) * eu * eu / T(2);
    }
    // fields first .. last-1 of direction q pulled from node s (one plane each)
    __device__ static void decode_fields(const S* __restrict__ Pin, const float4* __restrict__, long long ps, int q,
                                         int, int, int, T, int s, T (&v)[4], int first, int last)
    {
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (m >= first && m < last) v[m] = __ldg(Pin + off(m, q, ps, s));
    }
    __device__ static void store4(S* __restrict__ Pout, int q, long long ps, int g, const T (&v)[4], const T (&)[4])
    {
#pragma unroll
        for (int m = 0; m < 4; m++) Pout[off(m, q, ps, g)] = v[m];
    }
    // collide and store the four fields of direction q (collide_store's
    // operations, per field)
    __device__ static void collide_dir(S* __restrict__ Pout, int q, long long ps, int g, const T (&in)[4],
                                       const T (&r)[4], T pw, const T (&c1)[4], const T (&c2)[4], T w, T rt)
    {
        T o[4], f[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            f[m] = feq(r[m], pw, q, tiny(r[m]));
            o[m] = in[m] * c1[m] + c2[m] * f[m];
        }
        o[1] = o[1] - w * rt;
        o[2] = o[2] - w * rt;
        o[3] = o[3] + (w * rt) * T(2);
        store4(Pout, q, ps, g, o, f);
    }
};

// FP32 arithmetic and storage.
struct F32 {
    using T = float;
    using S = float;
    static constexpr bool kMoments = false;
    static constexpr bool kOnePass = true;
    // direction-major planes of ps nodes, the four fields of a node
    // interleaved: one 16-byte access moves a node's direction q
    __host__ __device__ static long long off(int fld, int q, long long ps, long long g)
    {
        return (((long long)q * ps + g) << 2) + fld;
    }
    __device__ static void load4(const S* p, T (&v)[4])
    {
        const float4 x = __ldg((const float4*)p);
        v[0] = x.x;
        v[1] = x.y;
        v[2] = x.z;
        v[3] = x.w;
    }
    __device__ static void encode4(S* p, const T (&v)[4], const T (&)[4])
    {
        *(float4*)p = make_float4(v[0], v[1], v[2], v[3]);
    }
    __device__ static void store4(S* Pout, int q, long long ps, int g, const T (&v)[4], const T (&feq)[4])
    {
        encode4(Pout + off(0, q, ps, g), v, feq);
    }
    // poly holds w_q * poly_q, so that an equilibrium value is one multiply
    __device__ static void poly(T ux, T uy, T uz, T (&p)[19])
    {
        const float omt = omt_term(ux, uy, uz);
#pragma unroll
        for (int q = 0; q < 19; q++) p[q] = __fmul_rn(poly_q_omt(q, ux, uy, uz, omt), (float)wq(q));
    }
    __device__ static bool tiny(T) { return false; }
    __device__ static T feq(T r, T pw, int, bool) { return r * pw; }
    // w * poly of one direction given by (ex, ey, ez) and weight w
    __device__ static T pw_dir(int ex, int ey, int ez, T w, T ux, T uy, T uz)
    {
        return __fmul_rn(poly_e_omt(ex, ey, ez, ux, uy, uz, omt_term(ux, uy, uz)), w);
    }
    // the four fields pulled from source s along (ex, ey, ez) of direction q,
    // as the pairs (flow, A), (B, C)
    __device__ static void decode_pairs(const S* __restrict__ Pin, const float4* __restrict__, long long ps, int q, int,
                                        int, int, T, int s, float2& v01, float2& v23)
    {
        const float4 x = __ldg((const float4*)(Pin + off(0, q, ps, s)));
        v01 = make_float2(x.x, x.y);
        v23 = make_float2(x.z, x.w);
    }
    // the stored bytes of (q, s): one 16-byte access
    using Raw = float4;
    __device__ static Raw load_raw(const S* __restrict__ Pin, long long ps, int q, int s)
    {
        return __ldg((const float4*)(Pin + off(0, q, ps, s)));
    }
    __device__ static void decode_raw(const Raw& x, int, int, int, T, const float4&, const float4&, float2& v01,
                                      float2& v23)
    {
        v01 = make_float2(x.x, x.y);
        v23 = make_float2(x.z, x.w);
    }
    __device__ static void decode_pairs_rec(const S* __restrict__ Pin, long long ps, int q, int ex, int ey, int ez,
                                            T w, int s, const float4& mf, const float4& ms, float2& v01, float2& v23)
    {
        decode_raw(load_raw(Pin, ps, q, s), ex, ey, ez, w, mf, ms, v01, v23);
    }
    __device__ static void decode4(const S* __restrict__ Pin, const float4* __restrict__, long long ps, int q, int,
                                   int, int, T, int s, T (&v)[4])
    {
        load4(Pin + off(0, q, ps, s), v);
    }
    __device__ static void store_pairs(S* Pout, int q, long long ps, int g, float2 o01, float2 o23, float2, float2)
    {
        *(float4*)(Pout + off(0, q, ps, g)) = make_float4(o01.x, o01.y, o23.x, o23.y);
    }
    // collide direction q of the four fields (collide_pairs) and store it
    __device__ static void collide_store(S* Pout, int q, long long ps, int g, float2 in01, float2 in23, float2 r01,
                                         float2 r23, float pw, float2 c1a, float2 c1b, float2 c2a, float2 c2b,
                                         float wrt)
    {
        float2 o01, o23, f01, f23;
        collide_pairs(in01, in23, r01, r23, pw, c1a, c1b, c2a, c2b, wrt, o01, o23, f01, f23);
        store_pairs(Pout, q, ps, g, o01, o23, f01, f23);
    }
    // collide and store the four fields of direction q (packed pairs)
    __device__ static void collide_dir(S* Pout, int q, long long ps, int g, const T (&in)[4], const T (&r)[4], T pw,
                                       const T (&c1)[4], const T (&c2)[4], T w, T rt)
    {
        collide_store(Pout, q, ps, g, make_float2(in[0], in[1]), make_float2(in[2], in[3]), make_float2(r[0], r[1]),
                      make_float2(r[2], r[3]), pw, make_float2(c1[0], c1[1]), make_float2(c1[2], c1[3]),
                      make_float2(c2[0], c2[1]), make_float2(c2[2], c2[3]), w * rt);
    }
    // fields first .. last-1 (one vector access brings all four)
    __device__ static void decode_fields(const S* __restrict__ Pin, const float4* __restrict__ M, long long ps, int q,
                                         int ex, int ey, int ez, T w, int s, T (&v)[4], int first, int last)
    {
        T u[4];
        decode4(Pin, M, ps, q, ex, ey, ez, w, s, u);
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (m >= first && m < last) v[m] = u[m];
    }
    __device__ static T decode(const S* p, int, int, const float4*, long long, int) { return __ldg(p); }
    __device__ static void encode(S* p, T v, T) { *p = v; }
};

// FP32 arithmetic; populations stored in FP16 as their non-equilibrium part
// n_q = f_q - feq_q(rho, u) of the node that wrote them, next to that node's
// FP32 moments M = {(rho, cA, cB, cC), (ux, uy, uz, 1 - 1.5|u|^2)}, one 32-byte
// record per node (float4 M[2g], M[2g+1]; the densities in field-pair order,
// so that a pair (rho, cA) or (cB, cC) is one register pair of the packed
// arithmetic).  A reader adds back feq_q of the writer's moments.  The stored
// quantity is of the order of the gradients, so FP16 keeps about FP32
// accuracy of f.
struct F16 {
    using T = float;
    using S = __half;
    static constexpr bool kMoments = true;
    static constexpr bool kOnePass = true;
    // layout of F32: one 8-byte access moves the four fields of (q, node)
    __host__ __device__ static long long off(int fld, int q, long long ps, long long g)
    {
        return (((long long)q * ps + g) << 2) + fld;
    }
    __device__ static void load4(const S* p, T (&v)[4])
    {
        const uint2 x = __ldg((const uint2*)p);
        const float2 lo = __half22float2(*(const __half2*)&x.x), hi = __half22float2(*(const __half2*)&x.y);
        v[0] = lo.x;
        v[1] = lo.y;
        v[2] = hi.x;
        v[3] = hi.y;
    }
    __device__ static void encode4(S* p, const T (&v)[4], const T (&feq)[4])
    {
        const __half2 lo = __floats2half2_rn(v[0] - feq[0], v[1] - feq[1]);
        const __half2 hi = __floats2half2_rn(v[2] - feq[2], v[3] - feq[3]);
        uint2 x;
        x.x = *(const unsigned*)&lo;
        x.y = *(const unsigned*)&hi;
        *(uint2*)p = x;
    }
    __device__ static void store4(S* Pout, int q, long long ps, int g, const T (&v)[4], const T (&feq)[4])
    {
        encode4(Pout + off(0, q, ps, g), v, feq);
    }
    // poly holds w_q * poly_q (rounded as below), so that an equilibrium
    // value is one multiply
    __device__ static void poly(T ux, T uy, T uz, T (&p)[19])
    {
        const float omt = omt_term(ux, uy, uz);
#pragma unroll
        for (int q = 0; q < 19; q++) p[q] = __fmul_rn(poly_q_omt(q, ux, uy, uz, omt), (float)wq(q));
    }
    __device__ static bool tiny(T) { return false; }
    __device__ static T feq(T r, T pw, int, bool) { return __fmul_rn(r, pw); }
    // w_q * poly_q of a writer from its moment record {(rho, c), (u, omt)}
    __device__ static T src_pw(int q, const float4& mf, const float4& ms)
    {
        return __fmul_rn(poly_q_omt(q, ms.x, ms.y, ms.z, ms.w), (float)wq(q));
    }
    __device__ static T pw_dir(int ex, int ey, int ez, T w, T ux, T uy, T uz)
    {
        return __fmul_rn(poly_e_omt(ex, ey, ez, ux, uy, uz, omt_term(ux, uy, uz)), w);
    }
    // the four fields pulled from source s along (ex, ey, ez) of direction q,
    // as the pairs (flow, A), (B, C): the stored part plus the writer's
    // equilibrium, each product and sum rounded on its own
    __device__ static void decode_pairs(const S* __restrict__ Pin, const float4* __restrict__ M, long long ps, int q,
                                        int ex, int ey, int ez, T w, int s, float2& v01, float2& v23)
    {
        const float4 mf = __ldg(M + 2 * (long long)s), ms = __ldg(M + 2 * (long long)s + 1);
        decode_pairs_rec(Pin, ps, q, ex, ey, ez, w, s, mf, ms, v01, v23);
    }
    // the stored bytes of (q, s): one 8-byte access
    using Raw = uint2;
    __device__ static Raw load_raw(const S* __restrict__ Pin, long long ps, int q, int s)
    {
        return __ldg((const uint2*)(Pin + off(0, q, ps, s)));
    }
    // the same with the writer's record {mf, ms} given
    __device__ static void decode_pairs_rec(const S* __restrict__ Pin, long long ps, int q, int ex, int ey, int ez,
                                            T w, int s, const float4& mf, const float4& ms, float2& v01, float2& v23)
    {
        decode_raw(load_raw(Pin, ps, q, s), ex, ey, ez, w, mf, ms, v01, v23);
    }
    // ... and with the stored bytes given
    __device__ static void decode_raw(const Raw& x, int ex, int ey, int ez, T w, const float4& mf, const float4& ms,
                                      float2& v01, float2& v23)
    {
        const float2 raw01 = __half22float2(*(const __half2*)&x.x), raw23 = __half22float2(*(const __half2*)&x.y);
        const float pw = __fmul_rn(poly_e_omt(ex, ey, ez, ms.x, ms.y, ms.z, ms.w), w);
        const float2 pp = make_float2(pw, pw);
        v01 = __ffma2_rn(make_float2(mf.x, mf.y), pp, raw01);
        v23 = __ffma2_rn(make_float2(mf.z, mf.w), pp, raw23);
    }
    __device__ static void decode4(const S* __restrict__ Pin, const float4* __restrict__ M, long long ps, int q,
                                   int ex, int ey, int ez, T w, int s, T (&v)[4])
    {
        float2 a, b;
        decode_pairs(Pin, M, ps, q, ex, ey, ez, w, s, a, b);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
    // collide direction q of the four fields and store the stored part of
    // the result, o - f with f = r * pw the node's own equilibrium, formed
    // directly: with o = in + c2 * (f - in) - the reaction terms,
    // o - f = c1 * (in - f) - the reaction terms (c1 = 1 - c2), one FMA on a
    // difference of the order of the non-equilibrium part, where forming o
    // first rounds an order-one value and then cancels it
    __device__ static void collide_store(S* Pout, int q, long long ps, int g, float2 in01, float2 in23, float2 r01,
                                         float2 r23, float pw, float2 c1a, float2 c1b, float2, float2, float wrt)
    {
        const float2 pp = make_float2(pw, pw);
        const float2 f01 = __fmul2_rn(r01, pp), f23 = __fmul2_rn(r23, pp);
        const float2 n01 = __ffma2_rn(c1a, __fadd2_rn(in01, make_float2(-f01.x, -f01.y)), make_float2(0.0f, -wrt));
        const float2 n23 =
            __ffma2_rn(c1b, __fadd2_rn(in23, make_float2(-f23.x, -f23.y)), make_float2(-wrt, 2.0f * wrt));
        const __half2 lo = __float22half2_rn(n01), hi = __float22half2_rn(n23);
        uint2 x;
        x.x = *(const unsigned*)&lo;
        x.y = *(const unsigned*)&hi;
        *(uint2*)(Pout + off(0, q, ps, g)) = x;
    }
    __device__ static void collide_dir(S* Pout, int q, long long ps, int g, const T (&in)[4], const T (&r)[4], T pw,
                                       const T (&c1)[4], const T (&c2)[4], T w, T rt)
    {
        collide_store(Pout, q, ps, g, make_float2(in[0], in[1]), make_float2(in[2], in[3]), make_float2(r[0], r[1]),
                      make_float2(r[2], r[3]), pw, make_float2(c1[0], c1[1]), make_float2(c1[2], c1[3]),
                      make_float2(c2[0], c2[1]), make_float2(c2[2], c2[3]), w * rt);
    }
    __device__ static void decode_fields(const S* __restrict__ Pin, const float4* __restrict__ M, long long ps, int q,
                                         int ex, int ey, int ez, T w, int s, T (&v)[4], int first, int last)
    {
        T u[4];
        decode4(Pin, M, ps, q, ex, ey, ez, w, s, u);
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (m >= first && m < last) v[m] = u[m];
    }
    __device__ static T decode(const S* p, int fld, int q, const float4* M, long long, int src)
    {
        const float4 mf = __ldg(M + 2 * (long long)src), ms = __ldg(M + 2 * (long long)src + 1);
        const float r = fld == 0 ? mf.x : (fld == 1 ? mf.y : (fld == 2 ? mf.z : mf.w));
        return __half2float(__ldg(p)) + feq(r, src_pw(q, mf, ms), q, false);
    }
    __device__ static void encode(S* p, T v, T feq) { *p = __float2half_rn(v - feq); }
};


// ---------------------------------------------------------------------------
// per-node physics: equilibrium -> collision -> store
// ---------------------------------------------------------------------------

// Per-field constants by selection (fld may be a run-time value; see box_nx).
__device__ __forceinline__ double pick_field(const double (&a)[4], int fld)
{
    return fld == 0 ? a[0] : (fld == 1 ? a[1] : (fld == 2 ? a[2] : a[3]));
}
__device__ __forceinline__ double pick_species(const double (&cin)[3][2], int fld, int n)
{
    return fld == 1 ? cin[0][n] : (fld == 2 ? cin[1][n] : cin[2][n]);
}

// Collide one field given its populations f, density r and the shared
// equilibrium polynomial, and store the result.  The reaction source of
// Tmixer.cpp:9697-9761: species A and B (fld 1, 2) lose (w_q*rt)*1.0, C gains
// (w_q*rt)*2.0 (molecular weights Ma = Mb = 1, Mp = 2, :9667).  fld may be a
// run-time value; the arithmetic is the same either way.  The FP64 form
// collides as the reference writes it, f*c1 + c2*feq; the FP32 and FP16-storage
// forms as f + c2*(feq - f), the form of collide_pairs.
template <class PR>
__device__ __forceinline__ void collide_store(typename PR::S* __restrict__ Pout, long long ps, int g, int fld,
                                              const typename PR::T (&f)[19], typename PR::T r,
                                              const typename PR::T (&poly)[19], const Phys& P, typename PR::T rt)
{
    using T = typename PR::T;
    const T c1 = T(pick_field(P.c1, fld)), c2 = T(pick_field(P.c2, fld));
    const bool tiny = PR::tiny(r);
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const T feq = PR::feq(r, poly[q], q, tiny);
        T v = PR::kOnePass ? f[q] + c2 * (feq - f[q]) : f[q] * c1 + c2 * feq;
        if (fld == 1 || fld == 2) v = v - T(wq(q)) * rt;
        if (fld == 3) v = v + (T(wq(q)) * rt) * T(2);
        PR::encode(Pout + PR::off(fld, q, ps, g), v, feq);
    }
}

// ---------------------------------------------------------------------------
// initial state: f = feq(rho0, 0) for the flow and 0 for the species
// (Tmixer.cpp:1544-1585, 1835-2018), then the first step's collision.
// ---------------------------------------------------------------------------
// Writes the state the first step reads: populations to X.pout, densities to
// X.rcur, moments (FP16 form) to X.mcur.
template <class PR>
__device__ __forceinline__ void init_node(const StepPtrs& X, const Geom& G, const Phys& P, double rho0d, int g)
{
    using T = typename PR::T;
    typename PR::S* Pout = (typename PR::S*)X.pout;
    T* R = (T*)X.rcur;
    double* Mac = X.mac;
    const long long ps = G.ps;
    const T rho0 = T(rho0d);
    T poly[19];
    PR::poly(T(0), T(0), T(0), poly);
    T f[19], z[19];
#pragma unroll
    for (int q = 0; q < 19; q++) {
        if constexpr (PR::kOnePass) {  // poly holds w_q * poly_q
            f[q] = PR::feq(rho0, poly[q], q, false);
            z[q] = T(0);
        } else {
            const T d = q == 0 ? T(3) : (q <= 6 ? T(18) : T(36));
            f[q] = (rho0 * poly[q]) / d;
            z[q] = (T(0) * poly[q]) / d;
        }
    }
    const T rt = T(P.rateconst) * T(0) * T(0);
    collide_store<PR>(Pout, ps, g, 0, f, rho0, poly, P, rt);
    collide_store<PR>(Pout, ps, g, 1, z, T(0), poly, P, rt);
    collide_store<PR>(Pout, ps, g, 2, z, T(0), poly, P, rt);
    collide_store<PR>(Pout, ps, g, 3, z, T(0), poly, P, rt);
    R[g] = rho0;
    R[ps + g] = T(0);
    R[2 * ps + g] = T(0);
    R[3 * ps + g] = T(0);
    Mac[g] = rho0d;
#pragma unroll
    for (int m = 1; m < 7; m++) Mac[m * ps + g] = 0.0;
    if (PR::kMoments) {
        X.mcur[2 * (long long)g] = make_float4((float)rho0, 0.f, 0.f, 0.f);  // rho0, no species
        X.mcur[2 * (long long)g + 1] = make_float4(0.f, 0.f, 0.f, omt_term(0.f, 0.f, 0.f));  // at rest
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

template <class PR>
__device__ __forceinline__ void bulk_load(const typename PR::S* __restrict__ Pin, const float4* __restrict__ M,
                                          long long ps, int fld, const Geom& G, int g, int i, int k, int sy, int sz,
                                          int iface, typename PR::T (&v)[19])
{
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int src = bulk_src(G, g, i, k, sy, sz, iface, q);
        v[q] = PR::decode(Pin + PR::off(fld, q, ps, src), fld, q, M, ps, src);
    }
}

// One interior node; boundary nodes are left to the boundary kernels.
template <class PR>
__device__ __forceinline__ void bulk_node(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g)
{
    using T = typename PR::T;
    const typename PR::S* __restrict__ Pin = (const typename PR::S*)X.pin;
    typename PR::S* __restrict__ Pout = (typename PR::S*)X.pout;
    const float4* __restrict__ M = X.mprev;
    const long long ps = G.ps;
    int b, i, j, k;
    decode(G, g, b, i, j, k);
    if (is_boundary(G, b, i, j, k)) return;
    const int sy = box_nx(G, b), sz = box_nx(G, b) * box_ny(G, b);
    const int iface = (b == 0 && j == 1) ? 1 : ((b == 1 && j == G.mny) ? 2 : 0);

    // flow: moments, equilibrium polynomial (shared by all four fields: they
    // use the flow velocity, Tmixer.cpp:1602-1830), collision
    T poly[19];
    T rho, ux, uy, uz;
    {
        T f[19];
        bulk_load<PR>(Pin, M, ps, 0, G, g, i, k, sy, sz, iface, f);
        rho = sum19(f);
        T sxm, sym, szm;
        momentum(f, sxm, sym, szm);
        ux = sxm / rho;
        uy = sym / rho;
        uz = szm / rho;
        PR::poly(ux, uy, uz, poly);
        collide_store<PR>(Pout, ps, g, 0, f, rho, poly, P, T(0));
    }
    // species A and B: the reaction needs both densities before either
    // collides, so their populations are loaded twice (the second time from
    // cache) rather than held in registers
    T ca, cb;
    {
        T a[19];
        bulk_load<PR>(Pin, M, ps, 1, G, g, i, k, sy, sz, iface, a);
        ca = sum19(a);
        bulk_load<PR>(Pin, M, ps, 2, G, g, i, k, sy, sz, iface, a);
        cb = sum19(a);
    }
    const T rt = T(P.rateconst) * ca * cb;
    T cc;
    {
        T a[19];
        bulk_load<PR>(Pin, M, ps, 1, G, g, i, k, sy, sz, iface, a);
        collide_store<PR>(Pout, ps, g, 1, a, ca, poly, P, rt);
        bulk_load<PR>(Pin, M, ps, 2, G, g, i, k, sy, sz, iface, a);
        collide_store<PR>(Pout, ps, g, 2, a, cb, poly, P, rt);
        bulk_load<PR>(Pin, M, ps, 3, G, g, i, k, sy, sz, iface, a);
        cc = sum19(a);
        collide_store<PR>(Pout, ps, g, 3, a, cc, poly, P, rt);
    }
    // densities the junction edges read next step (Tmixer.cpp:8609, :8851)
    if (b == 0 && j == 2 && (i == G.ia || i == G.ib)) {
        T* Rcur = (T*)X.rcur;
        Rcur[g] = rho;
        Rcur[ps + g] = ca;
        Rcur[2 * ps + g] = cb;
        Rcur[3 * ps + g] = cc;
    }
    if (PR::kMoments) {
        X.mcur[2 * (long long)g] = make_float4((float)rho, (float)ca, (float)cb, (float)cc);
        X.mcur[2 * (long long)g + 1] =
            make_float4((float)ux, (float)uy, (float)uz, omt_term((float)ux, (float)uy, (float)uz));
    }
    if (write_macro) {
        double* Mac = X.mac;
        Mac[g] = rho;
        Mac[ps + g] = ux;
        Mac[2 * ps + g] = uy;
        Mac[3 * ps + g] = uz;
        Mac[4 * ps + g] = ca;
        Mac[5 * ps + g] = cb;
        Mac[6 * ps + g] = cc;
    }
}

// Writer records of the FP16 form for lp_interior: read from global memory at
// the source node (the flat bulk kernel) ...
struct RecGlobal {
    const float4* __restrict__ M;
    __device__ __forceinline__ void operator()(int, int s, float4& mf, float4& ms) const
    {
        mf = __ldg(M + 2 * (long long)s);
        ms = __ldg(M + 2 * (long long)s + 1);
    }
};
// ... or from the shared-memory planes of a sweep tile (sweep_tile): plane
// slot (k - ez) & 3, row ty + 1 - ey, column tx + 1 - ex of (TY + 2) x 34
// records, the two halves of each record in separate arrays.
template <int TY>
struct RecShared {
    const float4* A;
    const float4* B;
    int tx, ty, k;
    __device__ __forceinline__ void operator()(int q, int, float4& mf, float4& ms) const
    {
        const int e = (((k - EZ(q)) & 3) * (TY + 2) + ty + 1 - EY(q)) * 34 + tx + 1 - EX(q);
        mf = A[e];
        ms = B[e];
    }
};

// The stored populations of a source for lp_interior, loaded from global
// memory.
template <class PR>
struct PopGlobal {
    const typename PR::S* __restrict__ Pin;
    long long ps;
    __device__ __forceinline__ typename PR::Raw operator()(int q, int s) const { return PR::load_raw(Pin, ps, q, s); }
};
// One interior node (b, i, j, k) = g for the reduced-precision forms (FP32
// arithmetic): every source index and (FP16 form) every writer's record
// (from rec) is fetched once per direction and all 76 populations decoded in
// one pass, which the FP32 register budget affords (the FP64 form loads field
// by field).  The arithmetic does not depend on where the records and the
// stored populations (pop) come from.
template <class PR, class Rec, class Pop>
__device__ __forceinline__ void lp_interior(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g,
                                            int b, int i, int j, int k, const Rec& rec, const Pop& pop)
{
    using T = typename PR::T;
    typename PR::S* __restrict__ Pout = (typename PR::S*)X.pout;
    const long long ps = G.ps;
    const int sy = box_nx(G, b), sz = box_nx(G, b) * box_ny(G, b);
    const int iface = (b == 0 && j == 1) ? 1 : ((b == 1 && j == G.mny) ? 2 : 0);

    // the four fields as the pairs (flow, A), (B, C)
    float2 p01[19], p23[19];
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int s = bulk_src(G, g, i, k, sy, sz, iface, q);
        float4 mf = make_float4(0.f, 0.f, 0.f, 0.f), ms = mf;
        if constexpr (PR::kMoments) rec(q, s, mf, ms);
        PR::decode_raw(pop(q, s), EX(q), EY(q), EZ(q), (float)wq(q), mf, ms, p01[q], p23[q]);
    }
    // sums in index order, two fields at a time
    float2 s01 = p01[0], s23 = p23[0];
#pragma unroll
    for (int q = 1; q < 19; q++) {
        s01 = __fadd2_rn(s01, p01[q]);
        s23 = __fadd2_rn(s23, p23[q]);
    }
    const T rho = s01.x, ca = s01.y, cb = s23.x, cc = s23.y;
    T f[19];
#pragma unroll
    for (int q = 0; q < 19; q++) f[q] = p01[q].x;
    T sxm, sym, szm;
    momentum(f, sxm, sym, szm);
    const T ux = sxm / rho, uy = sym / rho, uz = szm / rho;
    T poly[19];
    PR::poly(ux, uy, uz, poly);
    const T rt = T(P.rateconst) * ca * cb;
    const float2 r01 = make_float2(rho, ca), r23 = make_float2(cb, cc);
    const float2 c1a = make_float2((float)P.c1[0], (float)P.c1[1]), c1b = make_float2((float)P.c1[2], (float)P.c1[3]);
    const float2 c2a = make_float2((float)P.c2[0], (float)P.c2[1]), c2b = make_float2((float)P.c2[2], (float)P.c2[3]);
#pragma unroll
    for (int q = 0; q < 19; q++)
        PR::collide_store(Pout, q, ps, g, p01[q], p23[q], r01, r23, poly[q], c1a, c1b, c2a, c2b, (float)wq(q) * rt);
    if (b == 0 && j == 2 && (i == G.ia || i == G.ib)) {
        T* Rcur = (T*)X.rcur;
        Rcur[g] = rho;
        Rcur[ps + g] = ca;
        Rcur[2 * ps + g] = cb;
        Rcur[3 * ps + g] = cc;
    }
    if (PR::kMoments) {
        X.mcur[2 * (long long)g] = make_float4((float)rho, (float)ca, (float)cb, (float)cc);
        X.mcur[2 * (long long)g + 1] =
            make_float4((float)ux, (float)uy, (float)uz, omt_term((float)ux, (float)uy, (float)uz));
    }
    if (write_macro) {
        double* Mac = X.mac;
        Mac[g] = rho;
        Mac[ps + g] = ux;
        Mac[2 * ps + g] = uy;
        Mac[3 * ps + g] = uz;
        Mac[4 * ps + g] = ca;
        Mac[5 * ps + g] = cb;
        Mac[6 * ps + g] = cc;
    }
}


template <class T>
__device__ __forceinline__ void wall_flow_closure(int cls, T rout, T (&v)[19]);

// The z wall face node (b, i, j, kw), kw = 1 or nz (class K_FACE_Z1 or
// K_FACE_ZT), above or below interior node (b, i, j, kn), kn = 2 or nz - 1,
// which the calling thread of a sweep kernel has just updated.  Every z wall
// face node lies over an interior node and every interior node of planes 2
// and nz - 1 under one (boundary_list checks it), and with a sweep shape the
// boundary lists leave these nodes to the sweep kernels.  The node's flow is pulled from planes kw and kn
// and closed by the wall closure; its species are the interior neighbour's
// pulls (the zero-gradient copy).  The operations are those of
// boundary_lane_lp's four lanes for these classes (decode_raw, the closure,
// sum19, momentum, pw_dir, collide_dir), so the results equal the face
// kernel's bit for bit.  recw / recn give the writers' records of the wall
// node's and of the interior node's sources (FP16 form).
template <class PR, class Rec>
__device__ __forceinline__ void zwall_node(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int b,
                                           int i, int j, int kw, int kn, int gw, int gn, const Rec& recw,
                                           const Rec& recn)
{
    using T = typename PR::T;
    const typename PR::S* __restrict__ Pin = (const typename PR::S*)X.pin;
    typename PR::S* __restrict__ Pout = (typename PR::S*)X.pout;
    const long long ps = G.ps;
    const int sy = box_nx(G, b), sz = box_nx(G, b) * box_ny(G, b);
    const int iface = (b == 0 && j == 1) ? 1 : ((b == 1 && j == G.mny) ? 2 : 0);
    const int dz = kw == 1 ? 1 : -1;  // the lattice z component of the unknown directions
    const PopGlobal<PR> pop{Pin, ps};
    T f[19], a[19], bb[19], cc[19];
#pragma unroll
    for (int q = 0; q < 19; q++) {
        float4 mf = make_float4(0.f, 0.f, 0.f, 0.f), ms = mf;
        float2 v01, v23;
        const int s1 = bulk_src(G, gn, i, kn, sy, sz, iface, q);
        if constexpr (PR::kMoments) recn(q, s1, mf, ms);
        PR::decode_raw(pop(q, s1), EX(q), EY(q), EZ(q), (float)wq(q), mf, ms, v01, v23);
        a[q] = v01.y;
        bb[q] = v23.x;
        cc[q] = v23.y;
        f[q] = T(0);
        if (EZ(q) != dz) {
            const int s0 = bulk_src(G, gw, i, kw, sy, sz, iface, q);
            if constexpr (PR::kMoments) recw(q, s0, mf, ms);
            PR::decode_raw(pop(q, s0), EX(q), EY(q), EZ(q), (float)wq(q), mf, ms, v01, v23);
            f[q] = v01.x;
        }
    }
    wall_flow_closure(kw == 1 ? (int)K_FACE_Z1 : (int)K_FACE_ZT, T(P.rho_out), f);
    const T rho = sum19(f), ca = sum19(a), cb = sum19(bb), ccc = sum19(cc);
    T sxm, sym, szm;
    momentum(f, sxm, sym, szm);
    const T ux = sxm / rho, uy = sym / rho, uz = szm / rho;
    const T rt = T(P.rateconst) * ca * cb;
    const T rr[4] = {rho, ca, cb, ccc};
    T c1[4], c2[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        c1[m] = T(P.c1[m]);
        c2[m] = T(P.c2[m]);
    }
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const T in[4] = {f[q], a[q], bb[q], cc[q]};
        PR::collide_dir(Pout, q, ps, gw, in, rr, PR::pw_dir(EX(q), EY(q), EZ(q), (float)wq(q), ux, uy, uz), c1, c2,
                        (float)wq(q), rt);
    }
    T* __restrict__ Rcur = (T*)X.rcur;
    Rcur[gw] = rho;
    Rcur[ps + gw] = ca;
    Rcur[2 * ps + gw] = cb;
    Rcur[3 * ps + gw] = ccc;
    if constexpr (PR::kMoments) {
        X.mcur[2 * (long long)gw] = make_float4((float)rho, (float)ca, (float)cb, (float)ccc);
        X.mcur[2 * (long long)gw + 1] =
            make_float4((float)ux, (float)uy, (float)uz, omt_term((float)ux, (float)uy, (float)uz));
    }
    if (write_macro) {
        double* Mac = X.mac;
        Mac[gw] = rho;
        Mac[ps + gw] = ux;
        Mac[2 * ps + gw] = uy;
        Mac[3 * ps + gw] = uz;
        Mac[4 * ps + gw] = ca;
        Mac[5 * ps + gw] = cb;
        Mac[6 * ps + gw] = ccc;
    }
}

// One interior node of the FP32 / FP16 forms in the flat bulk kernels.  (The
// z wall faces stay with the face kernel here: updated by these kernels as
// well, the walls cost them registers (168 B of spills) and the 4-mixer FP16
// batch step went from 571 to 680-697 us, the W=32 FP16 step from 69.2 to
// 73.1 us.)
template <class PR>
__device__ __forceinline__ void bulk_node_lp(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g)
{
    int b, i, j, k;
    decode(G, g, b, i, j, k);
    if (is_boundary(G, b, i, j, k)) return;
    lp_interior<PR>(X, G, P, write_macro, g, b, i, j, k, RecGlobal{X.mprev},
                    PopGlobal<PR>{(const typename PR::S*)X.pin, G.ps});
}

// ---------------------------------------------------------------------------
// FP16 form, interior nodes by tiles (the sweep kernels).  A block of 32 x TY
// threads owns a tile of 32 x TY nodes of one box (x0.., y0..) and walks it
// through the planes z0 .. z1-1, one node per thread per plane.  The writer
// records its nodes read (the 9 source rows of each node, 19 reads per node in
// the flat kernel) are staged once per plane in shared memory: a ring of four
// planes of (TY + 2) x 34 records (the tile and a one-node halo), the next
// plane but one copied asynchronously (cp.async) while the current plane is
// computed.  The populations stream straight from global memory.  Each node's
// arithmetic is lp_interior's, so the results are the flat kernel's bit for
// bit.
// ---------------------------------------------------------------------------
constexpr int kSweepX = 32;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// The node whose record a tile of box b stages at 0-based (x, y) of plane kk:
// the node itself inside the box; on the inlet box's row y = -1 over the
// opening the mixing box's row mny, and on the mixing box's row y = mny the
// inlet box's row 1 (the sources of the two interface rules, as bulk_src);
// -1 where there is no node.
__device__ __forceinline__ int tile_rec_node(const Geom& G, int b, int x, int y, int kk)
{
    if (kk < 1 || kk > G.nz) return -1;
    const int nx = box_nx(G, b), ny = box_ny(G, b);
    if (x >= 0 && x < nx && y >= 0 && y < ny) return box_base(G, b) + ((kk - 1) * ny + y) * nx + x;
    if (b == 0 && y == -1) {
        const int xm = x - (G.ia - 1);
        if (xm >= 0 && xm < G.mnx) return G.base[1] + ((kk - 1) * G.mny + (G.mny - 1)) * G.mnx + xm;
    } else if (b == 1 && y == G.mny) {
        const int xi = x + G.ia - 1;
        if (xi >= 0 && xi < G.inx) return ((kk - 1) * G.iny) * G.inx + xi;
    }
    return -1;
}

// One tile {mixer * 2 + box, x0 | y0 << 16, z0 | z1 << 16} (0-based x0, y0;
// interior planes z0 .. z1-1, 2 <= z0 < z1 <= nz).  A and B hold the two
// halves of 4 * (TY + 2) * 34 records.  Every thread of the block runs the
// same iterations (the barriers are uniform).  The tiles of the first chunk
// (z0 = 2) also update the z = 1 wall face nodes of their columns, those of
// the last chunk (z1 = nz) the z = nz ones (zwall_node), the records of
// both planes being in the ring.
template <class PR, int TY>
__device__ __forceinline__ void sweep_tile(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int4 t,
                                           float4* A, float4* B)
{
    constexpr int RW = kSweepX + 2, PLANE = (TY + 2) * RW, NT = kSweepX * TY;
    const int b = t.x & 1;
    const int x0 = t.y & 0xffff, y0 = t.y >> 16, z0 = t.z & 0xffff, z1 = t.z >> 16;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int nx = box_nx(G, b), ny = box_ny(G, b);
    const int x = x0 + tx, y = y0 + ty;
    const float4* __restrict__ M = X.mprev;
    auto stage = [&](int kk) {
        const int slot = (kk & 3) * PLANE;
        for (int e = threadIdx.x; e < PLANE; e += NT) {
            const int ry = e / RW, rx = e - ry * RW;
            const int n = tile_rec_node(G, b, x0 + rx - 1, y0 + ry - 1, kk);
            if (n >= 0) {
                cp_async16(A + slot + e, M + 2 * (long long)n);
                cp_async16(B + slot + e, M + 2 * (long long)n + 1);
            }
        }
    };
    stage(z0 - 1);
    stage(z0);
    stage(z0 + 1);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    for (int k = z0; k < z1; k++) {
        // plane k + 2 goes to the slot of plane k - 2, which no thread reads
        // any more (the barrier at the end of the previous iteration)
        if (k + 2 < z1 + 1) stage(k + 2);
        cp_async_commit();
        if (x < nx && y < ny && !is_boundary(G, b, x + 1, y + 1, k)) {
            const int g = box_base(G, b) + ((k - 1) * ny + y) * nx + x;
            lp_interior<PR>(X, G, P, write_macro, g, b, x + 1, y + 1, k, RecShared<TY>{A, B, tx, ty, k},
                            PopGlobal<PR>{(const typename PR::S*)X.pin, G.ps});
            if (k == 2)
                zwall_node<PR>(X, G, P, write_macro, b, x + 1, y + 1, 1, 2, g - nx * ny, g,
                               RecShared<TY>{A, B, tx, ty, 1}, RecShared<TY>{A, B, tx, ty, 2});
            if (k == G.nz - 1)
                zwall_node<PR>(X, G, P, write_macro, b, x + 1, y + 1, G.nz, k, g + nx * ny, g,
                               RecShared<TY>{A, B, tx, ty, G.nz}, RecShared<TY>{A, B, tx, ty, k});
        }
        cp_async_wait_all();
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// boundary closures (Tmixer.cpp:2023-9033)
// ---------------------------------------------------------------------------
template <class PR>
struct BCtx {
    using T = typename PR::T;
    const typename PR::S* __restrict__ Pin;
    const float4* __restrict__ M;  // writers' moments (FP16 form)
    const T* __restrict__ Rprev;
    const T* __restrict__ uin1;
    const T* __restrict__ uin2;
    const Geom* G;
    const Phys* P;
    long long ps;
    int g, b, i, j, k;
};

template <class PR>
__device__ __forceinline__ typename PR::T own_fn(const BCtx<PR>& c, int fld, int q)
{
    return PR::decode(c.Pin + PR::off(fld, q, c.ps, c.g), fld, q, c.M, c.ps, c.g);
}
template <class PR>
__device__ __forceinline__ typename PR::T rprev(const BCtx<PR>& c, int fld, int b, int i, int j, int k)
{
    return __ldg(c.Rprev + (long long)fld * c.ps + node_index(*c.G, b, i, j, k));
}
template <class PR>
__device__ __forceinline__ typename PR::T uin(const BCtx<PR>& c, int side, int j, int k)
{
    return __ldg((side == 0 ? c.uin1 : c.uin2) + j * (c.G->nz + 3) + k);
}
template <class PR>
__device__ __forceinline__ void pull_node(const BCtx<PR>& c, int fld, int b, int i, int j, int k,
                                          typename PR::T (&v)[19])
{
    using T = typename PR::T;
#pragma unroll
    for (int q = 0; q < 19; q++) {
        const int s = pull_src(*c.G, b, i, j, k, q);
        v[q] = s >= 0 ? PR::decode(c.Pin + PR::off(fld, q, c.ps, s), fld, q, c.M, c.ps, s) : T(0);
    }
}
// the same sum as sum19 without two directions (the closures' "rho - (...)")
template <class T>
__device__ __forceinline__ T sum_but(const T (&v)[19], int a, int d)
{
    T s = T(0);
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
template <class PR>
__device__ __forceinline__ typename PR::T inlet_rho_now(const BCtx<PR>& c, int side, int j, int k)
{
    using T = typename PR::T;
    T v[19];
    const int x = side == 0 ? 1 : c.G->inx;
    pull_node(c, 0, 0, x, j, k, v);
    const T U = uin(c, side, j, k);
    if (side == 0)
        return (T(1) / (T(1) - U)) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                    T(2) * (v[3] + v[8] + v[9] + v[12] + v[13]));
    return (T(1) / (T(1) + (U))) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                  T(2) * (v[1] + v[7] + v[10] + v[11] + v[14]));
}

// corners: six bounce-backs, buried pairs averaged from their own
// post-collision values, and (corners 1-12) one pair closed from a density.
struct CornerSpec {
    signed char bb[6][2];
    signed char navg;
    signed char avg[3][2];
    signed char cp[2];
};
static __constant__ CornerSpec kCorner[16] = {
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
template <class PR>
__device__ __forceinline__ void corner_closure(const BCtx<PR>& c, int fld, int n, typename PR::T R, typename PR::T* t)
{
    using T = typename PR::T;
    const CornerSpec& s = kCorner[n];
    for (int m = 0; m < 6; m++) t[s.bb[m][0]] = t[s.bb[m][1]];
    T fa[3];
    for (int m = 0; m < s.navg; m++) fa[m] = T(0.5) * (own_fn(c, fld, s.avg[m][0]) + own_fn(c, fld, s.avg[m][1]));
    for (int m = 0; m < s.navg; m++) {
        t[s.avg[m][0]] = fa[m];
        t[s.avg[m][1]] = fa[m];
    }
    if (s.cp[0] >= 0) {
        T sum = T(0);
        bool first = true;
        for (int q = 0; q < 19; q++) {
            if (q == s.cp[0] || q == s.cp[1]) continue;
            sum = first ? t[q] : sum + t[q];
            first = false;
        }
        t[s.cp[0]] = T(0.5) * (R - sum);
        t[s.cp[1]] = t[s.cp[0]];
    }
}

// Flow closures of the y and z walls, the outlet and the mixing box's x walls
// on a node's pulled populations (the species of these faces are a copy of
// the interior neighbour's pulls).
template <class T>
__device__ __forceinline__ void wall_flow_closure(int cls, T rout, T (&v)[19])
{
    switch (cls) {
    case K_FACE_YT: {  // Case 10 flow (:2731-2764); species copy from y-1 (:2766-2872)
        const T C = T(0.5) * (v[5] - v[6] + v[11] + v[12] - v[13] - v[14]);
        v[4] = v[2]; v[16] = v[18] - C; v[17] = v[15] + C;
        const T A = T(0.5) * (v[1] - v[3] + v[11] - v[12] - v[13] + v[14]);
        v[9] = v[7] + A; v[10] = v[8] - A;
    } break;
    case K_FACE_Y1: {  // Cases 11, 12 flow (:2874-2906, :3016-3049); species copy from y+1
        const T C = T(0.5) * (v[5] - v[6] + v[11] + v[12] - v[13] - v[14]);
        v[2] = v[4]; v[15] = v[17] - C; v[18] = v[16] + C;
        const T A = T(0.5) * (v[1] - v[3] + v[11] - v[12] - v[13] + v[14]);
        v[7] = v[9] - A; v[8] = v[10] + A;
    } break;
    case K_OUTLET: {  // Case 13 flow (:3162-3190); species copy from y+1 (:3192-3273)
        const T uy = T(1) - (T(1) / rout) * ((v[0] + v[1] + v[3] + v[5] + v[6] + v[11] + v[12] + v[13] + v[14]) +
                                                T(2) * (v[4] + v[9] + v[10] + v[16] + v[17]));
        const T A = (rout * uy) / T(6);
        const T B = T(0.5) * ((v[3] + v[12] + v[13]) - (v[1] + v[11] + v[14]));
        const T C = T(0.5) * ((v[6] + v[13] + v[14]) - (v[5] + v[11] + v[12]));
        v[2] = v[4] + (rout * uy) / T(3);
        v[7] = v[9] + (A + B); v[8] = v[10] + (A - B); v[15] = v[17] + (A + C); v[18] = v[16] + (A - C);
    } break;
    case K_FACE_MX1: {  // Case 14 (:3275-3404); species copy from x+1
        const T C = T(0.5) * ((v[6] + v[17] + v[18]) - (v[5] + v[15] + v[16]));
        v[1] = v[3]; v[11] = v[13] + (C); v[14] = v[12] - (C);
        const T A = T(0.5) * ((v[2] + v[15] + v[18]) - (v[4] + v[16] + v[17]));
        v[7] = v[9] - A; v[10] = v[8] + A;
    } break;
    case K_FACE_MXT: {  // Case 15 (:3405-3539); species copy from x-1
        const T C = T(0.5) * ((v[6] + v[17] + v[18]) - (v[5] + v[15] + v[16]));
        v[3] = v[1]; v[13] = v[11] - (C); v[12] = v[14] + (C);
        const T A = T(0.5) * ((v[2] + v[15] + v[18]) - (v[4] + v[16] + v[17]));
        v[9] = v[7] + A; v[8] = v[10] - A;
    } break;
    case K_FACE_ZT: {  // Cases 16, 17 and the opening nodes of 17 (:3540-3887); species copy from z-1
        const T B = T(0.5) * (v[2] - v[4] + v[7] + v[8] - v[9] - v[10]);
        v[6] = v[5]; v[17] = v[15] + B; v[18] = v[16] - B;
        const T A = T(0.5) * (v[1] - v[3] + v[7] - v[8] - v[9] + v[10]);
        v[13] = v[11] + A; v[14] = v[12] - A;
    } break;
    case K_FACE_Z1: {  // Cases 18, 19 and the opening nodes of 19 (:3888-4237); species copy from z+1
        const T B = T(0.5) * (v[2] - v[4] + v[7] + v[8] - v[9] - v[10]);
        v[5] = v[6]; v[15] = v[17] - B; v[16] = v[18] + B;
        const T A = T(0.5) * (v[1] - v[3] + v[7] - v[8] - v[9] + v[10]);
        v[11] = v[13] - A; v[12] = v[14] + A;
    } break;
    default: break;
    }
}

// Apply the closure of class `cls` to field fld of the node in c, on v (the
// node's pulled populations).  Closures follow the reference case by case;
// the comments give the reference lines.  Face classes (inlets, outlet, walls)
// and edge/corner classes are separate functions so that each boundary kernel
// holds only the code of its own classes.
template <class PR>
__device__ __forceinline__ void closure_face(const BCtx<PR>& c, int cls, int fld, typename PR::T (&v)[19])
{
    using T = typename PR::T;
    const bool flow = fld == 0;
    switch (cls) {
    case K_INLET1: {  // Inlet1 (:2606-2666)
        if (flow) {
            const T U = uin(c, 0, c.j, c.k);
            const T r = (T(1) / (T(1) - U)) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                                  T(2) * (v[3] + v[8] + v[9] + v[12] + v[13]));
            const T A = (-r * U) / T(6);
            const T B = T(0.5) * (v[2] - v[4] + v[15] - v[16] - v[17] + v[18]);
            const T C = T(0.5) * (v[5] - v[6] + v[15] + v[16] - v[17] - v[18]);
            v[1] = v[3] + (r * U) / T(3);
            v[7] = v[9] - (A + B); v[10] = v[8] - (A - B); v[11] = v[13] - (A + C); v[14] = v[12] - (A - C);
        } else {
            const T cin = pick_species(c.P->cin, fld, 0);
            v[1] = -v[3] + T(2.0 / 18.0) * cin;
            v[7] = -v[9] + T(2.0 / 36.0) * cin;
            v[10] = -v[8] + T(2.0 / 36.0) * cin;
            v[11] = -v[13] + T(2.0 / 36.0) * cin;
            v[14] = -v[12] + T(2.0 / 36.0) * cin;
        }
    } break;
    case K_INLET2: {  // Inlet2 (:2668-2730)
        if (flow) {
            const T U = uin(c, 1, c.j, c.k);
            const T r = (T(1) / (T(1) + (U))) * ((v[0] + v[2] + v[4] + v[5] + v[6] + v[15] + v[16] + v[17] + v[18]) +
                                                    T(2) * (v[1] + v[7] + v[10] + v[11] + v[14]));
            const T A = (-r * (U)) / T(6);
            const T B = T(0.5) * (v[2] - v[4] + v[15] - v[16] - v[17] + v[18]);
            const T C = T(0.5) * (v[5] - v[6] + v[15] + v[16] - v[17] - v[18]);
            v[3] = v[1] - (r * (U)) / T(3);
            v[9] = v[7] + (A + B); v[8] = v[10] + (A - B); v[13] = v[11] + (A + C); v[12] = v[14] + (A - C);
        } else {
            const T cin = pick_species(c.P->cin, fld, 1);
            v[3] = -v[1] + T(2.0 / 18.0) * cin;
            v[9] = -v[7] + T(2.0 / 36.0) * cin;
            v[8] = -v[10] + T(2.0 / 36.0) * cin;
            v[13] = -v[11] + T(2.0 / 36.0) * cin;
            v[12] = -v[14] + T(2.0 / 36.0) * cin;
        }
    } break;
    case K_FACE_YT:
    case K_FACE_Y1:
    case K_OUTLET:
    case K_FACE_MX1:
    case K_FACE_MXT:
    case K_FACE_ZT:
    case K_FACE_Z1:
        // the species of these faces are copied from the interior neighbour
        // by the pull itself (face_copy_offset); only the flow is closed
        if (flow) wall_flow_closure(cls, T(c.P->rho_out), v);
        break;
    default: break;
    }
}

template <class PR>
__device__ __forceinline__ void closure_edge(const BCtx<PR>& c, int cls, int fld, typename PR::T (&v)[19])
{
    using T = typename PR::T;
    const Geom& G = *c.G;
    const bool flow = fld == 0;
    switch (cls) {
    case K_EDGE_Y1_ZTOP: {  // Cases 2, 3 (:2030-2342)
        v[2] = v[4]; v[6] = v[5]; v[7] = v[9]; v[8] = v[10]; v[13] = v[11]; v[14] = v[12]; v[18] = v[16];
        v[15] = T(0.5) * (own_fn(c, fld, 15) + own_fn(c, fld, 17));
        v[17] = v[15];
        const T A = T(0.25) * (v[1] - v[3]);
        v[7] = v[9] - A; v[8] = v[10] + A; v[13] = v[11] + A; v[14] = v[12] - A;
    } break;
    case K_EDGE_X1_ZTOP: {  // Case 4 (:2343-2476); field C keeps p13 = pn13 (:2474)
        const T B = T(0.25) * (v[2] - v[4]);
        v[1] = v[3]; v[6] = v[5]; v[7] = v[9] - B; v[10] = v[8] + B; v[14] = v[12]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[13] = own_fn(c, fld, 13);
        v[11] = T(0.5) * (rprev(c, fld, 0, 1, c.j, G.nz - 1) - sum_but(v, 11, 13));
        if (fld != 3) v[13] = v[11];
    } break;
    case K_EDGE_XT_ZTOP: {  // Case 6 (:2477-2605)
        const T B = T(0.25) * (v[2] - v[4]);
        v[3] = v[1]; v[6] = v[5]; v[9] = v[7] + B; v[8] = v[10] - B; v[13] = v[11]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[12] = T(0.5) * (rprev(c, fld, 0, G.inx, c.j, G.nz - 1) - sum_but(v, 12, 14));
        v[14] = v[12];
    } break;
    case K_EDGE_YT_ZT: {  // Case 20 (:4238-4385)
        v[4] = v[2]; v[6] = v[5]; v[17] = v[15];
        v[16] = T(0.5) * (own_fn(c, fld, 16) + own_fn(c, fld, 18));
        v[18] = v[16];
        const T A = T(0.25) * (v[1] - v[3]);
        v[9] = v[7] + A; v[10] = v[8] - A; v[13] = v[11] + A; v[14] = v[12] - A;
    } break;
    case K_EDGE_YT_Z1: {  // Case 21 (:4386-4533)
        v[4] = v[2]; v[5] = v[6]; v[16] = v[18];
        v[15] = T(0.5) * (own_fn(c, fld, 15) + own_fn(c, fld, 17));
        v[17] = v[15];
        const T A = T(0.25) * (v[1] - v[3]);
        v[9] = v[7] + A; v[10] = v[8] - A; v[11] = v[13] - A; v[12] = v[14] + A;
    } break;
    case K_EDGE_X1_Z1: {  // Case 22 (:4534-4656); flow density of (1,j,2) from this step
        const T B = T(0.25) * (v[2] - v[4]);
        v[1] = v[3]; v[5] = v[6]; v[7] = v[9] - B; v[10] = v[8] + B; v[11] = v[13]; v[15] = v[17] - B; v[16] = v[18] + B;
        const T R = flow ? inlet_rho_now(c, 0, c.j, 2) : rprev(c, fld, 0, 1, c.j, 2);
        v[12] = T(0.5) * (R - sum_but(v, 12, 14));
        v[14] = v[12];
    } break;
    case K_EDGE_XT_Z1: {  // Case 23 (:4657-4779)
        const T B = T(0.25) * (v[2] - v[4]);
        v[3] = v[1]; v[5] = v[6]; v[8] = v[10] - B; v[9] = v[7] + B; v[12] = v[14]; v[15] = v[17] - B; v[16] = v[18] + B;
        const T R = flow ? inlet_rho_now(c, 1, c.j, 2) : rprev(c, fld, 0, G.inx, c.j, 2);
        v[11] = T(0.5) * (R - sum_but(v, 11, 13));
        v[13] = v[11];
    } break;
    case K_EDGE_X1_Y1: {  // Case 24 (:4780-4909)
        const T C = T(0.25) * (v[5] - v[6]);
        v[1] = v[3]; v[2] = v[4]; v[7] = v[9]; v[11] = v[13] - C; v[14] = v[12] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const T R = flow ? inlet_rho_now(c, 0, 2, c.k) : rprev(c, fld, 0, 1, 2, c.k);
        v[8] = T(0.5) * (R - sum_but(v, 8, 10));
        v[10] = v[8];
    } break;
    case K_EDGE_X1_YT: {  // Case 25 (:4910-5032)
        const T C = T(0.25) * (v[5] - v[6]);
        v[1] = v[3]; v[4] = v[2]; v[10] = v[8]; v[11] = v[13] - C; v[14] = v[12] + C; v[16] = v[18] - C; v[17] = v[15] + C;
        const T R = flow ? inlet_rho_now(c, 0, G.iny - 1, c.k) : rprev(c, fld, 0, 1, G.iny - 1, c.k);
        v[7] = T(0.5) * (R - sum_but(v, 7, 9));
        v[9] = v[7];
    } break;
    case K_EDGE_XT_Y1: {  // Case 26 (:5033-5159)
        const T C = T(0.25) * (v[5] - v[6]);
        v[3] = v[1]; v[2] = v[4]; v[8] = v[10]; v[12] = v[14] - C; v[13] = v[11] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const T R = flow ? inlet_rho_now(c, 1, 2, c.k) : rprev(c, fld, 0, G.inx, 2, c.k);
        v[7] = T(0.5) * (R - sum_but(v, 7, 9));
        v[9] = v[7];
    } break;
    case K_EDGE_XT_YT: {  // Case 27 (:5160-5281)
        const T C = T(0.25) * (v[5] - v[6]);
        v[3] = v[1]; v[4] = v[2]; v[9] = v[7]; v[12] = v[14] - C; v[13] = v[11] + C; v[16] = v[18] - C; v[17] = v[15] + C;
        const T R = flow ? inlet_rho_now(c, 1, G.iny - 1, c.k) : rprev(c, fld, 0, G.inx, G.iny - 1, c.k);
        v[8] = T(0.5) * (R - sum_but(v, 8, 10));
        v[10] = v[8];
    } break;
    case K_EDGE_Y1_Z1: {  // Cases 28, 29 (:5282-5571)
        v[2] = v[4]; v[5] = v[6]; v[15] = v[17];
        v[16] = T(0.5) * (own_fn(c, fld, 16) + own_fn(c, fld, 18));
        v[18] = v[16];
        const T A = T(0.25) * (v[1] - v[3]);
        v[7] = v[9] - A; v[8] = v[10] + A; v[11] = v[13] - A; v[12] = v[14] + A;
    } break;
    case K_MEDGE_AB: {  // (:7788-7868)
        const T A = T(0.25) * (v[1] - v[3]);
        v[2] = v[4]; v[5] = v[6]; v[7] = v[9] - A; v[8] = v[10] + A; v[11] = v[13] - A; v[12] = v[14] + A; v[15] = v[17];
        const T R = flow ? T(c.P->rho_out) : rprev(c, fld, 1, c.i, 2, 1);
        v[18] = T(0.5) * (R - sum_but(v, 16, 18));
        v[16] = v[18];
    } break;
    case K_MEDGE_ApBp: {  // (:7870-7950)
        const T A = T(0.25) * (v[1] - v[3]);
        v[2] = v[4]; v[6] = v[5]; v[7] = v[9] - A; v[8] = v[10] + A; v[13] = v[11] + A; v[14] = v[12] - A; v[18] = v[16];
        const T R = flow ? T(c.P->rho_out) : rprev(c, fld, 1, c.i, 2, G.nz);
        v[15] = T(0.5) * (R - sum_but(v, 15, 17));
        v[17] = v[15];
    } break;
    case K_MEDGE_AAp: {  // (:7951-8043)
        const T C = T(0.25) * (v[5] - v[6]);
        v[1] = v[3]; v[2] = v[4]; v[7] = v[9]; v[11] = v[13] - C; v[14] = v[12] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const T R = flow ? T(c.P->rho_out) : rprev(c, fld, 1, 1, 2, c.k);
        v[8] = T(0.5) * (R - sum_but(v, 8, 10));
        v[10] = v[8];
    } break;
    case K_MEDGE_BBp: {  // (:8044-8136)
        const T C = T(0.25) * (v[5] - v[6]);
        v[3] = v[1]; v[2] = v[4]; v[8] = v[10]; v[12] = v[14] - C; v[13] = v[11] + C; v[15] = v[17] - C; v[18] = v[16] + C;
        const T R = flow ? T(c.P->rho_out) : rprev(c, fld, 1, G.mnx, 2, c.k);
        v[7] = T(0.5) * (R - sum_but(v, 7, 9));
        v[9] = v[7];
    } break;
    case K_MEDGE_AD: {  // (:8137-8244)
        const T B = T(0.25) * (v[2] - v[4]);
        v[1] = v[3]; v[5] = v[6]; v[7] = v[9] - B; v[10] = v[8] + B; v[11] = v[13]; v[15] = v[17] - B; v[16] = v[18] + B;
        v[14] = T(0.5) * (own_fn(c, fld, 12) + own_fn(c, fld, 14));
        v[12] = v[14];
    } break;
    case K_MEDGE_ApDp: {  // (:8245-8344)
        const T B = T(0.25) * (v[2] - v[4]);
        v[1] = v[3]; v[6] = v[5]; v[7] = v[9] - B; v[10] = v[8] + B; v[14] = v[12]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[13] = T(0.5) * (own_fn(c, fld, 11) + own_fn(c, fld, 13));
        v[11] = v[13];
    } break;
    case K_MEDGE_BC: {  // (:8345-8445)
        const T B = T(0.25) * (v[2] - v[4]);
        v[3] = v[1]; v[5] = v[6]; v[8] = v[10] - B; v[9] = v[7] + B; v[12] = v[14]; v[15] = v[17] - B; v[16] = v[18] + B;
        v[13] = T(0.5) * (own_fn(c, fld, 11) + own_fn(c, fld, 13));
        v[11] = v[13];
    } break;
    case K_MEDGE_BpCp: {  // (:8446-8550)
        const T B = T(0.25) * (v[2] - v[4]);
        v[3] = v[1]; v[6] = v[5]; v[9] = v[7] + B; v[8] = v[10] - B; v[13] = v[11]; v[17] = v[15] + B; v[18] = v[16] - B;
        v[14] = T(0.5) * (own_fn(c, fld, 12) + own_fn(c, fld, 14));
        v[12] = v[14];
    } break;
    case K_JUNC_DD:    // (:8551-8792): closed pair 7/9 from the density at (ia, 2, k)
    case K_JUNC_CC: {  // (:8793-9033): closed pair 8/10 from the density at (ib, 2, k)
        const bool dd = cls == K_JUNC_DD;
        T a;
        a = T(0.5) * (own_fn(c, fld, 3) + own_fn(c, fld, 1)); v[3] = a; v[1] = a;
        a = T(0.5) * (own_fn(c, fld, 4) + own_fn(c, fld, 2)); v[4] = a; v[2] = a;
        a = T(0.5) * (own_fn(c, fld, 5) + own_fn(c, fld, 6)); v[6] = a; v[5] = a;
        a = T(0.5) * (own_fn(c, fld, 11) + own_fn(c, fld, 13)); v[13] = a; v[11] = a;
        a = T(0.5) * (own_fn(c, fld, 12) + own_fn(c, fld, 14)); v[14] = a; v[12] = a;
        a = T(0.5) * (own_fn(c, fld, 15) + own_fn(c, fld, 17)); v[17] = a; v[15] = a;
        a = T(0.5) * (own_fn(c, fld, 16) + own_fn(c, fld, 18)); v[18] = a; v[16] = a;
        const T R = rprev(c, fld, 0, dd ? G.ia : G.ib, 2, c.k);
        if (dd) {
            a = T(0.5) * (own_fn(c, fld, 8) + own_fn(c, fld, 10)); v[10] = a; v[8] = a;
            v[7] = T(0.5) * (R - sum_but(v, 7, 9));
            v[9] = v[7];
        } else {
            a = T(0.5) * (own_fn(c, fld, 7) + own_fn(c, fld, 9)); v[9] = a; v[7] = a;
            v[8] = T(0.5) * (R - sum_but(v, 8, 10));
            v[10] = v[8];
        }
    } break;
    default: {
        if (cls >= K_CORNER_1 && cls <= K_CORNER_16) {
            const int n = cls - K_CORNER_1;
            T R = T(0);
            if (n < 8) {  // inlet corners: density of the adjacent x-y edge node
                R = rprev(c, fld, 0, c.i, c.j, c.k == G.nz ? G.nz - 1 : 2);
            } else if (n < 12) {  // outlet corners: rho_out; species read the row
                R = flow ? T(c.P->rho_out) : T(0);  // below the outlet, which is 0
            }
            T t[19];
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
// The interior neighbour whose pulled species populations a face node copies
// (zero-gradient closure), or (0, 0, 0) for a face without that closure.
__device__ __forceinline__ void face_copy_offset(int cls, int& di, int& dj, int& dk)
{
    di = dj = dk = 0;
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
}

template <class PR, bool FACES>
__device__ __forceinline__ void closed_pull(const BCtx<PR>& c, int cls, int fld, typename PR::T (&v)[19])
{
    // one pull for the four lanes, the species lanes of a copy class from
    // the interior neighbour: the warp runs the 19 pulls once, not once per
    // branch
    int di = 0, dj = 0, dk = 0;
    if (FACES && fld > 0) face_copy_offset(cls, di, dj, dk);
    pull_node(c, fld, c.b, c.i + di, c.j + dj, c.k + dk, v);
    if (di | dj | dk) return;
    if (FACES)
        closure_face(c, cls, fld, v);
    else
        closure_edge(c, cls, fld, v);
}

// One wall face node (wall_class) in one thread, the four fields in the
// order of bulk_node: the flow pulled and closed, then the species copied from
// the interior neighbour's pulls (A and B summed first for the reaction term,
// then pulled again to collide, then C).  The arithmetic is boundary_lane's:
// the same sums, moments, outlet density, polynomial and collision.  One loop
// over the six passes keeps a single copy of the pull and collision code.
template <class PR>
__device__ __forceinline__ void wall_node(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g,
                                          int b, int i, int j, int k, int cls)
{
    using T = typename PR::T;
    const typename PR::S* __restrict__ Pin = (const typename PR::S*)X.pin;
    typename PR::S* __restrict__ Pout = (typename PR::S*)X.pout;
    const long long ps = G.ps;
    int di, dj, dk;
    face_copy_offset(cls, di, dj, dk);
    T poly[19];
    T rho = T(0), ux = T(0), uy = T(0), uz = T(0), ca = T(0), cb = T(0), cc = T(0), rt = T(0);
#pragma unroll 1
    for (int s = 0; s < 6; s++) {
        const int fld = s == 0 ? 0 : (s < 3 ? s : (s < 5 ? s - 2 : 3));  // flow, A, B, A, B, C
        const int o = fld ? 1 : 0;
        T v[19];
#pragma unroll
        for (int q = 0; q < 19; q++) {
            const int src = pull_src(G, b, i + o * di, j + o * dj, k + o * dk, q);
            v[q] = src >= 0 ? PR::decode(Pin + PR::off(fld, q, ps, src), fld, q, nullptr, ps, src) : T(0);
        }
        if (s == 0) wall_flow_closure(cls, T(P.rho_out), v);
        T r = sum19(v);
        if (s == 0) {
            // the outlet row's density is pinned to rho_out (Tmixer.cpp:9575-9582)
            if (b == 1 && j == 1) r = T(P.rho_out);
            T sxm, sym, szm;
            momentum(v, sxm, sym, szm);
            ux = sxm / r;
            uy = sym / r;
            uz = szm / r;
            PR::poly(ux, uy, uz, poly);
            rho = r;
        } else if (s == 1) {
            ca = r;
            continue;
        } else if (s == 2) {
            cb = r;
            rt = T(P.rateconst) * ca * cb;
            continue;
        }
        if (s == 5) cc = r;
        collide_store<PR>(Pout, ps, g, fld, v, s == 3 ? ca : (s == 4 ? cb : r), poly, P, rt);
    }
    T* __restrict__ Rcur = (T*)X.rcur;
    Rcur[g] = rho;
    Rcur[ps + g] = ca;
    Rcur[2 * ps + g] = cb;
    Rcur[3 * ps + g] = cc;
    if (write_macro) {
        double* Mac = X.mac;
        Mac[g] = rho;
        Mac[ps + g] = ux;
        Mac[2 * ps + g] = uy;
        Mac[3 * ps + g] = uz;
        Mac[4 * ps + g] = ca;
        Mac[5 * ps + g] = cb;
        Mac[6 * ps + g] = cc;
    }
}

// ---------------------------------------------------------------------------
// boundary nodes of a compact, class-sorted list, four threads per node: lane
// fld (0 flow, 1 A, 2 B, 3 C) pulls, closes and collides its own field.  Every
// closure reads only its own field, so the lanes need each other only for
// the moments: the flow lane's density and velocity and the species
// densities (for the reaction term), passed by warp shuffles.  FACES selects
// the list of inlet/outlet/wall-face nodes or of edge/corner nodes.
// ---------------------------------------------------------------------------
constexpr int kBoundaryThreads = 128;
constexpr int kBoundaryLanes = 4;

// Lane fld of boundary node g (class cls); mask holds the active lanes of
// the warp and lead the first lane of this node's group of four.
template <class PR, bool FACES>
__device__ __forceinline__ void boundary_lane(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g,
                                              int cls, int fld, unsigned mask, int lead)
{
    using T = typename PR::T;
    typename PR::S* __restrict__ Pout = (typename PR::S*)X.pout;
    T* __restrict__ Rcur = (T*)X.rcur;
    double* __restrict__ Mac = X.mac;
    BCtx<PR> c;
    c.Pin = (const typename PR::S*)X.pin;
    c.M = X.mprev;
    c.Rprev = (const T*)X.rprev;
    c.uin1 = (const T*)X.uin1;
    c.uin2 = (const T*)X.uin2;
    c.G = &G;
    c.P = &P;
    c.ps = G.ps;
    c.g = g;
    decode(G, c.g, c.b, c.i, c.j, c.k);
    const long long ps = G.ps;

    T v[19];
    closed_pull<PR, FACES>(c, cls, fld, v);
    T r = sum19(v);
    T ux = T(0), uy = T(0), uz = T(0);
    if (fld == 0) {
        // the outlet row's density is pinned to rho_out (Tmixer.cpp:9575-9582)
        if (c.b == 1 && c.j == 1) r = T(P.rho_out);
        T sxm, sym, szm;
        momentum(v, sxm, sym, szm);
        ux = sxm / r;
        uy = sym / r;
        uz = szm / r;
    }
    ux = __shfl_sync(mask, ux, lead);
    uy = __shfl_sync(mask, uy, lead);
    uz = __shfl_sync(mask, uz, lead);
    const T rho = __shfl_sync(mask, r, lead);
    const T ca = __shfl_sync(mask, r, lead + 1);
    const T cb = __shfl_sync(mask, r, lead + 2);
    const T cc = __shfl_sync(mask, r, lead + 3);
    T poly[19];
    PR::poly(ux, uy, uz, poly);
    const T rt = fld == 0 ? T(0) : T(P.rateconst) * ca * cb;
    collide_store<PR>(Pout, ps, c.g, fld, v, r, poly, P, rt);

    Rcur[fld * ps + c.g] = r;
    if (PR::kMoments) {
        if (fld == 0) X.mcur[2 * (long long)c.g] = make_float4((float)rho, (float)ca, (float)cb, (float)cc);
        if (fld == 1)
            X.mcur[2 * (long long)c.g + 1] =
                make_float4((float)ux, (float)uy, (float)uz, omt_term((float)ux, (float)uy, (float)uz));
    }
    if (write_macro) {
        Mac[(fld == 0 ? 0 : 3 + fld) * ps + c.g] = r;
        if (fld == 0) {
            Mac[ps + c.g] = ux;
            Mac[2 * ps + c.g] = uy;
            Mac[3 * ps + c.g] = uz;
        }
    }
}

// Direction 4K + lane of a group of four lanes (K a compile-time constant,
// lane a run-time value): its lattice vector and weight, selected from the
// compile-time tables.  Returns false past direction 18.
template <int K>
__device__ __forceinline__ bool lane_dir(int lane, int& q, int& ex, int& ey, int& ez, double& w)
{
    constexpr int q0 = 4 * K, q1 = 4 * K + 1 < 19 ? 4 * K + 1 : 18, q2 = 4 * K + 2 < 19 ? 4 * K + 2 : 18,
                  q3 = 4 * K + 3 < 19 ? 4 * K + 3 : 18;
    q = q0 + lane;
    ex = lane == 0 ? EX(q0) : lane == 1 ? EX(q1) : lane == 2 ? EX(q2) : EX(q3);
    ey = lane == 0 ? EY(q0) : lane == 1 ? EY(q1) : lane == 2 ? EY(q2) : EY(q3);
    ez = lane == 0 ? EZ(q0) : lane == 1 ? EZ(q1) : lane == 2 ? EZ(q2) : EZ(q3);
    w = wq(q < 19 ? q : 18);
    return q < 19;
}

// Boundary node g with its four lanes splitting the work three ways:
//   1. directions: lane l pulls directions l, l+4, ... for all four fields
//      (one vector load, one moment record and one polynomial per
//      direction), species of a zero-gradient face from the interior
//      neighbour, into the node's 76-value buffer in shared memory;
//   2. fields: lane fld closes field fld (the same closures as
//      boundary_lane) and forms its density; moments by shuffle;
//   3. directions again: collide and store the four fields of each of its
//      directions with one vector store.
// Every value is computed with the operations, in the order, of the
// one-field-per-thread step (pull_node, the closures, sum19, momentum,
// collide_store), so the FP64 form stays bit-exact.
template <class PR, bool FACES>
__device__ __forceinline__ void boundary_lane_lp(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro,
                                                 int g, int cls, int fld, unsigned mask, int lead,
                                                 typename PR::T* buf)
{
    using T = typename PR::T;
    const typename PR::S* __restrict__ Pin = (const typename PR::S*)X.pin;
    typename PR::S* __restrict__ Pout = (typename PR::S*)X.pout;
    T* __restrict__ Rcur = (T*)X.rcur;
    double* __restrict__ Mac = X.mac;
    BCtx<PR> c;
    c.Pin = Pin;
    c.M = X.mprev;
    c.Rprev = (const T*)X.rprev;
    c.uin1 = (const T*)X.uin1;
    c.uin2 = (const T*)X.uin2;
    c.G = &G;
    c.P = &P;
    c.ps = G.ps;
    c.g = g;
    decode(G, c.g, c.b, c.i, c.j, c.k);
    const long long ps = G.ps;
    int di = 0, dj = 0, dk = 0;
    if (FACES) face_copy_offset(cls, di, dj, dk);
    const bool copy = (di | dj | dk) != 0;

    // 1. pull by direction
#define TMX_LANE_PULL(K)                                                                                         \
    {                                                                                                            \
        int q, ex, ey, ez;                                                                                       \
        double w;                                                                                                \
        if (lane_dir<K>(fld, q, ex, ey, ez, w)) {                                                                \
            T v[4] = {T(0), T(0), T(0), T(0)};                                                                   \
            const int s0 = pull_src_e(G, c.b, c.i, c.j, c.k, ex, ey, ez);                                        \
            /* a zero-gradient face takes its species from the interior neighbour */                             \
            if (s0 >= 0) PR::decode_fields(Pin, c.M, ps, q, ex, ey, ez, T(w), s0, v, 0, copy ? 1 : 4);           \
            if (copy) {                                                                                          \
                const int s1 = pull_src_e(G, c.b, c.i + di, c.j + dj, c.k + dk, ex, ey, ez);                     \
                if (s1 >= 0) PR::decode_fields(Pin, c.M, ps, q, ex, ey, ez, T(w), s1, v, 1, 4);                  \
            }                                                                                                    \
            buf[q] = v[0];                                                                                       \
            buf[19 + q] = v[1];                                                                                  \
            buf[38 + q] = v[2];                                                                                  \
            buf[57 + q] = v[3];                                                                                  \
        }                                                                                                        \
    }
    TMX_LANE_PULL(0)
    TMX_LANE_PULL(1)
    TMX_LANE_PULL(2)
    TMX_LANE_PULL(3)
    TMX_LANE_PULL(4)
#undef TMX_LANE_PULL
    __syncwarp(mask);

    // 2. close by field
    T v[19];
#pragma unroll
    for (int q = 0; q < 19; q++) v[q] = buf[fld * 19 + q];
    if (!(copy && fld > 0)) {
        if (FACES)
            closure_face(c, cls, fld, v);
        else
            closure_edge(c, cls, fld, v);
    }
    T r = sum19(v);
    T ux = T(0), uy = T(0), uz = T(0);
    if (fld == 0) {
        // the outlet row's density is pinned to rho_out (Tmixer.cpp:9575-9582)
        if (c.b == 1 && c.j == 1) r = T(P.rho_out);
        T sxm, sym, szm;
        momentum(v, sxm, sym, szm);
        ux = sxm / r;
        uy = sym / r;
        uz = szm / r;
    }
    ux = __shfl_sync(mask, ux, lead);
    uy = __shfl_sync(mask, uy, lead);
    uz = __shfl_sync(mask, uz, lead);
    const T rho = __shfl_sync(mask, r, lead);
    const T ca = __shfl_sync(mask, r, lead + 1);
    const T cb = __shfl_sync(mask, r, lead + 2);
    const T cc = __shfl_sync(mask, r, lead + 3);
#pragma unroll
    for (int q = 0; q < 19; q++) buf[fld * 19 + q] = v[q];
    __syncwarp(mask);

    // 3. collide and store by direction
    const T rt = T(P.rateconst) * ca * cb;
    const T rr[4] = {rho, ca, cb, cc};
    T c1[4], c2[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        c1[m] = T(P.c1[m]);
        c2[m] = T(P.c2[m]);
    }
#define TMX_LANE_STORE(K)                                                                                        \
    {                                                                                                            \
        int q, ex, ey, ez;                                                                                       \
        double w;                                                                                                \
        if (lane_dir<K>(fld, q, ex, ey, ez, w)) {                                                                \
            const T in[4] = {buf[q], buf[19 + q], buf[38 + q], buf[57 + q]};                                     \
            PR::collide_dir(Pout, q, ps, c.g, in, rr, PR::pw_dir(ex, ey, ez, T(w), ux, uy, uz), c1, c2, T(w), rt); \
        }                                                                                                        \
    }
    TMX_LANE_STORE(0)
    TMX_LANE_STORE(1)
    TMX_LANE_STORE(2)
    TMX_LANE_STORE(3)
    TMX_LANE_STORE(4)
#undef TMX_LANE_STORE

    Rcur[fld * ps + c.g] = r;
    if (PR::kMoments) {
        if (fld == 0) X.mcur[2 * (long long)c.g] = make_float4((float)rho, (float)ca, (float)cb, (float)cc);
        if (fld == 1)
            X.mcur[2 * (long long)c.g + 1] =
                make_float4((float)ux, (float)uy, (float)uz, omt_term((float)ux, (float)uy, (float)uz));
    }
    if (write_macro) {
        Mac[(fld == 0 ? 0 : 3 + fld) * ps + c.g] = r;
        if (fld == 0) {
            Mac[ps + c.g] = ux;
            Mac[2 * ps + c.g] = uy;
            Mac[3 * ps + c.g] = uz;
        }
    }
}

// Lane fld of boundary node g in the form's scheme: directions split across
// the lanes for the interleaved forms (buf: the node's 76 values of shared
// memory); one field per lane for FP64, whose SoA planes give the direction
// split no saving and whose larger code then stalls on instruction fetch
// (65.5 us against 59.6 us for the W=32 faces).
template <class PR, bool FACES>
__device__ __forceinline__ void boundary_any(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g,
                                             int cls, int fld, unsigned mask, int lead, typename PR::T* buf)
{
    if constexpr (PR::kOnePass)
        boundary_lane_lp<PR, FACES>(X, G, P, write_macro, g, cls, fld, mask, lead, buf);
    else
        boundary_lane<PR, FACES>(X, G, P, write_macro, g, cls, fld, mask, lead);
}

// One launch over a node list: thread 4t + fld is lane fld of node t.
template <class PR, bool FACES>
__device__ __forceinline__ void boundary_node(const StepPtrs& X, const int* __restrict__ bnode,
                                              const unsigned char* __restrict__ bcls, int nb, const Geom& G,
                                              const Phys& P, int write_macro, typename PR::T (*buf)[76], int blk)
{
    const int gt = blk * blockDim.x + threadIdx.x;
    const int t = gt >> 2, fld = gt & 3;
    // the four lanes of a node share one warp; whole nodes drop out together
    const unsigned mask = __ballot_sync(0xffffffffu, t < nb);
    if (t >= nb) return;
    boundary_any<PR, FACES>(X, G, P, write_macro, bnode[t], bcls[t], fld, mask, (threadIdx.x & 31) & ~3,
                            buf[threadIdx.x >> 2]);
}

// One interior node in the form's bulk scheme: one pass over the 76 values
// for the interleaved layouts, field by field for FP64.
template <class PR>
__device__ __forceinline__ void bulk_any(const StepPtrs& X, const Geom& G, const Phys& P, int write_macro, int g)
{
    if constexpr (PR::kOnePass)
        bulk_node_lp<PR>(X, G, P, write_macro, g);
    else
        bulk_node<PR>(X, G, P, write_macro, g);
}

// Kernel definitions for one precision policy; NAME is the kernel-name suffix.
#define TMX_DEFINE_STEP_KERNELS(PR, NAME)                                                                         \
    __global__ void k_init_##NAME(StepPtrs X, Geom G, Phys P, double rho0)                                      \
    {                                                                                                           \
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G.nnodes; g += gridDim.x * blockDim.x)          \
            init_node<PR>(X, G, P, rho0, g);                                                                    \
    }                                                                                                           \
    __global__ void __launch_bounds__(256, 2) k_bulk_##NAME(StepPtrs X, Geom G, Phys P, int write_macro)        \
    {                                                                                                           \
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G.nnodes; g += gridDim.x * blockDim.x)          \
            bulk_any<PR>(X, G, P, write_macro, g);                                                              \
    }

// A batched kernel's block works on one mixer at a time (a sweep tile, 32
// entries of a boundary list).  The block copies what the step reads of that
// mixer's descriptor (the buffers of this step's parity, the geometry, the
// physics) to shared memory, between two barriers of the caller, and the
// step code reads them from there: read through a reference into the global
// descriptor array, the compiler reloaded them from global memory inside the
// node loop (about 60 extra global loads per interior node of the sweep
// kernel, which cost it 12% of its time).  The flat interior kernel keeps
// the global descriptor: its two barriers per cell block cost more than the
// reloads.
struct StepDesc {
    StepPtrs X;
    Geom G;
    Phys P;
};
__device__ __forceinline__ void load_desc(StepDesc& dst, const MixerDesc* __restrict__ D, int m, int parity)
{
    static_assert(sizeof(StepPtrs) % 8 == 0 && sizeof(Geom) % 8 == 0 && sizeof(Phys) % 8 == 0 &&
                      sizeof(StepDesc) == sizeof(StepPtrs) + sizeof(Geom) + sizeof(Phys),
                  "descriptor copied in 8-byte words");
    constexpr int nx = sizeof(StepPtrs) / 8, nw = sizeof(StepDesc) / 8;
    const unsigned long long* __restrict__ sx = (const unsigned long long*)&D[m].X[parity];
    const unsigned long long* __restrict__ sg = (const unsigned long long*)&D[m].G;
    unsigned long long* d = (unsigned long long*)&dst;
    for (int e = threadIdx.x; e < nw; e += blockDim.x) d[e] = e < nx ? __ldg(sx + e) : __ldg(sg + (e - nx));
}

// The FP16 form's interior as tiles (sweep_tile), persistent over the tile
// list: 32 x 8 threads (two blocks per SM) or 32 x 4 (four).  Dynamic shared
// memory: sweep_smem_host(TY).
#define TMX_SWEEP_KERNEL(PR, NAME, TY, MINB)                                                                      \
    __global__ void __launch_bounds__(kSweepX * TY, MINB) k_sweep##TY##_##NAME(                                  \
        StepPtrs X, Geom G, Phys P, int write_macro, const int4* __restrict__ tiles, int ntiles)                 \
    {                                                                                                           \
        extern __shared__ float4 sweep_smem[];                                                                  \
        float4* A = sweep_smem;                                                                                 \
        float4* B = A + 4 * (TY + 2) * (kSweepX + 2);                                                           \
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) sweep_tile<PR, TY>(X, G, P, write_macro, tiles[t], A, B); \
    }                                                                                                           \
    __global__ void __launch_bounds__(kSweepX * TY, MINB) k_sweep_batch##TY##_##NAME(                            \
        const MixerDesc* __restrict__ D, const int4* __restrict__ tiles, const int* __restrict__ counts,         \
        int parity, int write_macro)                                                                            \
    {                                                                                                           \
        extern __shared__ float4 sweep_smem[];                                                                  \
        float4* A = sweep_smem;                                                                                 \
        float4* B = A + 4 * (TY + 2) * (kSweepX + 2);                                                           \
        __shared__ StepDesc d;                                                                                  \
        const int n = counts[3];                                                                                \
        for (int t = blockIdx.x; t < n; t += gridDim.x) {                                                       \
            const int4 tl = tiles[t];                                                                           \
            __syncthreads();                                                                                    \
            load_desc(d, D, tl.x >> 1, parity);                                                                 \
            __syncthreads();                                                                                    \
            sweep_tile<PR, TY>(d.X, d.G, d.P, write_macro, tl, A, B);                                           \
        }                                                                                                       \
    }
#define TMX_DEFINE_SWEEP_KERNELS(PR, NAME) \
    TMX_SWEEP_KERNEL(PR, NAME, 8, 2)       \
    TMX_SWEEP_KERNEL(PR, NAME, 4, 4)

// The face and the edge list as two launches (the FP32 and FP16-storage steps;
// the FP64 step uses k_bound and k_walls).
#define TMX_DEFINE_BOUNDARY_KERNELS(PR, NAME)                                                                     \
    __global__ void __launch_bounds__(kBoundaryThreads) k_bfaces_##NAME(                                       \
        StepPtrs X, const int* bnode, const unsigned char* bcls, int nb, Geom G, Phys P, int write_macro)       \
    {                                                                                                           \
        __shared__ PR::T buf[PR::kOnePass ? kBoundaryThreads / 4 : 1][76];                                      \
        boundary_node<PR, true>(X, bnode, bcls, nb, G, P, write_macro, buf, blockIdx.x);                        \
    }                                                                                                           \
    __global__ void __launch_bounds__(kBoundaryThreads) k_bedges_##NAME(                                       \
        StepPtrs X, const int* bnode, const unsigned char* bcls, int nb, Geom G, Phys P, int write_macro)       \
    {                                                                                                           \
        __shared__ PR::T buf[PR::kOnePass ? kBoundaryThreads / 4 : 1][76];                                      \
        boundary_node<PR, false>(X, bnode, bcls, nb, G, P, write_macro, buf, blockIdx.x);                       \
    }

// Faces and edges in one launch, the first eblocks blocks on the edge and
// corner list (bnode + nf), the rest on the face list (the FP64 step, whose
// bulk kernel follows the boundary).
#define TMX_DEFINE_BOUND_KERNEL(PR, NAME)                                                                         \
    __global__ void __launch_bounds__(kBoundaryThreads) k_bound_##NAME(StepPtrs X, const int* bnode,           \
        const unsigned char* bcls, int nf, int ne, int eblocks, Geom G, Phys P, int write_macro)                 \
    {                                                                                                           \
        __shared__ PR::T buf[PR::kOnePass ? kBoundaryThreads / 4 : 1][76];                                      \
        if ((int)blockIdx.x < eblocks)                                                                          \
            boundary_node<PR, false>(X, bnode + nf, bcls + nf, ne, G, P, write_macro, buf, blockIdx.x);         \
        else                                                                                                    \
            boundary_node<PR, true>(X, bnode, bcls, nf, G, P, write_macro, buf, blockIdx.x - eblocks);          \
    }

// The wall faces (wall_class), one thread per node of a node-sorted list.
#define TMX_DEFINE_WALL_KERNEL(PR, NAME)                                                                          \
    __global__ void __launch_bounds__(kBoundaryThreads) k_walls_##NAME(StepPtrs X, const int* wnode,           \
        const unsigned char* wcls, int nw, Geom G, Phys P, int write_macro)                                     \
    {                                                                                                           \
        const int t = blockIdx.x * blockDim.x + threadIdx.x;                                                    \
        if (t >= nw) return;                                                                                    \
        const int g = wnode[t];                                                                                 \
        int b, i, j, k;                                                                                         \
        decode(G, g, b, i, j, k);                                                                               \
        wall_node<PR>(X, G, P, write_macro, g, b, i, j, k, wcls[t]);                                            \
    }


// Batched kernels for one precision policy (declared in tmx_kernels.cuh).
#define TMX_BULK_BATCH(PR, NAME, NT)                                                                              \
    __global__ void __launch_bounds__(NT, 512 / NT) k_bulk_batch##NT##_##NAME(                                  \
        const MixerDesc* __restrict__ D, const int4* __restrict__ blocks, const int* __restrict__ counts,        \
        int parity, int write_macro)                                                                            \
    {                                                                                                           \
        const int nblk = counts[0];                                                                             \
        for (int b = blockIdx.x; b < nblk; b += gridDim.x) {                                                    \
            const int4 cb = blocks[b];                                                                          \
            const MixerDesc& d = D[cb.x];                                                                       \
            for (int t = threadIdx.x; t < cb.z; t += NT) bulk_any<PR>(d.X[parity], d.G, d.P, write_macro, cb.y + t); \
        }                                                                                                       \
    }
// The batched boundary kernels hold the shared descriptor's values in
// registers; their register counts are held to those of the global-descriptor
// build (72 and 80 for the interleaved forms' faces and edges, 128 for FP64),
// which kept them at 7, 6 and 4 blocks per SM: the 4-mixer FP16 sweep step
// took 511-517 us capped against 528-533 us uncapped.
#define TMX_BOUNDARY_BATCH(PR, NAME, KIND, FACES, WHICH)                                                          \
    __global__ void __launch_bounds__(kBoundaryThreads, PR::kOnePass ? (FACES ? 7 : 6) : 4)                    \
        k_##KIND##_batch_##NAME(                                                                                \
        const MixerDesc* __restrict__ D, const int2* __restrict__ list, const int* __restrict__ counts,         \
        int parity, int write_macro)                                                                            \
    {                                                                                                           \
        const int n = counts[WHICH];                                                                            \
        __shared__ PR::T buf[PR::kOnePass ? kBoundaryThreads / 4 : 1][76];                                      \
        __shared__ StepDesc d;                                                                                  \
        for (int base = blockIdx.x * blockDim.x; base < 4 * n; base += gridDim.x * blockDim.x) {                \
            const int t = (base + threadIdx.x) >> 2, fld = threadIdx.x & 3;                                     \
            /* entries base / 4 .. base / 4 + 31 belong to one mixer (kListAlign) */                            \
            __syncthreads();                                                                                    \
            load_desc(d, D, list[base >> 2].y >> 8, parity);                                                    \
            __syncthreads();                                                                                    \
            const int2 e = t < n ? list[t] : make_int2(-1, 0);                                                  \
            const bool live = e.x >= 0;                                                                         \
            const unsigned mask = __ballot_sync(0xffffffffu, live);                                             \
            if (live)                                                                                           \
                boundary_any<PR, FACES>(d.X, d.G, d.P, write_macro, e.x, e.y & 255, fld, mask,                  \
                                        (threadIdx.x & 31) & ~3, buf[threadIdx.x >> 2]);                        \
        }                                                                                                       \
    }
#define TMX_DEFINE_BATCH_KERNELS(PR, NAME)        \
    TMX_BULK_BATCH(PR, NAME, 128)                 \
    TMX_BULK_BATCH(PR, NAME, 256)                 \
    TMX_BULK_BATCH(PR, NAME, 512)                 \
    TMX_BOUNDARY_BATCH(PR, NAME, bfaces, true, 1) \
    TMX_BOUNDARY_BATCH(PR, NAME, bedges, false, 2)

}  // namespace tmx
