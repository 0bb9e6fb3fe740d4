// tmx_probe.cu -- the memory-traffic ceiling of the interior kernels' access
// pattern (benchmark support; no counterpart in the reference).
//
// A lattice update of the interior kernels reads 19 direction planes, each at
// a node shifted by its lattice vector, and writes the same 19 planes at the
// node itself: 38 concurrent streams per form (FP64: 76 planes of doubles, one
// per field and direction; FP32: 19 planes of the four fields as 16 bytes;
// FP16: 19 planes of 8 bytes plus the node's 32-byte moment record read and
// written).  These kernels move exactly those bytes, in those layouts, with no
// arithmetic.  Their throughput is what DRAM gives this pattern, as opposed to
// the two streams of a plain copy; an interior kernel's achieved bandwidth
// over it says how much of the pattern's own ceiling the kernel reaches.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/tmx.h"
#include "tmx_host.h"

namespace {

using tmx_host::fail;

// lattice vectors of the 19 directions, in the reference's numbering
// (Tmixer.cpp:1368-1370)
constexpr int kEX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
constexpr int kEY[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
constexpr int kEZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};

// node offset of each direction's upstream neighbour in an x-fastest box
struct Offsets {
    int o[19];
};

constexpr int kThreads = 256;

// A stored value made to depend on every loaded value of the node (zero is 0
// at run time, which the compiler cannot know): all loads of a node are in
// flight before its first store, as in the step, instead of each store
// following its own load.
__device__ __forceinline__ double dep(double v, unsigned mix, int zero)
{
    return __longlong_as_double(__double_as_longlong(v) ^ (long long)(mix & (unsigned)zero));
}
__device__ __forceinline__ float4 dep(float4 v, unsigned mix, int zero)
{
    v.x = __uint_as_float(__float_as_uint(v.x) ^ (mix & (unsigned)zero));
    return v;
}
__device__ __forceinline__ uint2 dep(uint2 v, unsigned mix, int zero)
{
    v.x ^= mix & (unsigned)zero;
    return v;
}

// nodes lo .. hi-1 of ps; every upstream node g - o[q] lies in 0 .. ps-1
__global__ void __launch_bounds__(kThreads) k_pattern_f64(const double* __restrict__ in, double* __restrict__ out,
                                                         long long ps, int lo, int hi, Offsets off, int zero)
{
    for (int g = lo + blockIdx.x * blockDim.x + threadIdx.x; g < hi; g += gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 4; f++) {
            double v[19];
#pragma unroll
            for (int q = 0; q < 19; q++) v[q] = __ldg(in + (f * 19 + q) * ps + (g - off.o[q]));
            unsigned mix = 0;
#pragma unroll
            for (int q = 0; q < 19; q++) mix ^= (unsigned)__double_as_longlong(v[q]);
#pragma unroll
            for (int q = 0; q < 19; q++) out[(f * 19 + q) * ps + g] = dep(v[q], mix, zero);
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_pattern_f32(const float4* __restrict__ in, float4* __restrict__ out,
                                                         long long ps, int lo, int hi, Offsets off, int zero)
{
    for (int g = lo + blockIdx.x * blockDim.x + threadIdx.x; g < hi; g += gridDim.x * blockDim.x) {
        float4 v[19];
#pragma unroll
        for (int q = 0; q < 19; q++) v[q] = __ldg(in + q * ps + (g - off.o[q]));
        unsigned mix = 0;
#pragma unroll
        for (int q = 0; q < 19; q++) mix ^= __float_as_uint(v[q].x);
#pragma unroll
        for (int q = 0; q < 19; q++) out[q * ps + g] = dep(v[q], mix, zero);
    }
}

__global__ void __launch_bounds__(kThreads) k_pattern_f16(const uint2* __restrict__ in, uint2* __restrict__ out,
                                                         const float4* __restrict__ min, float4* __restrict__ mout,
                                                         long long ps, int lo, int hi, Offsets off, int zero)
{
    for (int g = lo + blockIdx.x * blockDim.x + threadIdx.x; g < hi; g += gridDim.x * blockDim.x) {
        uint2 v[19];
#pragma unroll
        for (int q = 0; q < 19; q++) v[q] = __ldg(in + q * ps + (g - off.o[q]));
        const float4 a = __ldg(min + 2 * (long long)g), b = __ldg(min + 2 * (long long)g + 1);
        unsigned mix = __float_as_uint(a.x) ^ __float_as_uint(b.x);
#pragma unroll
        for (int q = 0; q < 19; q++) mix ^= v[q].x;
#pragma unroll
        for (int q = 0; q < 19; q++) out[q * ps + g] = dep(v[q], mix, zero);
        mout[2 * (long long)g] = a;
        mout[2 * (long long)g + 1] = b;
    }
}

// device buffers, stream and events of one probe, released on every return
// path
struct Buffers {
    void* p[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    ~Buffers()
    {
        if (st) cudaStreamSynchronize(st);
        for (void* q : p)
            if (q) cudaFree(q);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (st) cudaStreamDestroy(st);
    }
};

}  // namespace

extern "C" int tmx_pattern_ceiling(int precision, long long nodes, int reps, int device, double* gbs,
                                   int* blocks_per_sm)
{
    if (!gbs) return fail(TMX_E_INVALID, "null argument");
    if (precision != TMX_FP64 && precision != TMX_FP32 && precision != TMX_FP16)
        return fail(TMX_E_INVALID, "unknown precision %d", precision);
    if (reps < 1) return fail(TMX_E_INVALID, "reps must be positive (got %d)", reps);
    // an x-fastest box 256 x 128 x nz holding at least `nodes` nodes
    const int nx = 256, ny = 128;
    const long long plane = (long long)nx * ny;
    if (nodes < 3 * plane || nodes > (1LL << 30))
        return fail(TMX_E_INVALID, "nodes must lie in [%lld, %lld] (got %lld)", 3 * plane, 1LL << 30, nodes);
    const long long nz = (nodes + plane - 1) / plane;
    const long long ps = plane * nz;
    // the nodes whose every upstream neighbour lies in the box
    const int lo = (int)(plane + nx + 1), hi = (int)(ps - plane - nx - 1);
    Offsets off;
    for (int q = 0; q < 19; q++) off.o[q] = kEX[q] + kEY[q] * nx + kEZ[q] * (int)plane;
    const long long pbytes = precision == TMX_FP64 ? 76 * 8 * ps : 19 * (precision == TMX_FP32 ? 16 : 8) * ps;
    const long long bytes_per_node = precision == TMX_FP64 ? 1216 : precision == TMX_FP32 ? 608 : 368;

    TMX_CK(cudaSetDevice(device));
    int sms = 0;
    TMX_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    Buffers buf;
    TMX_CK(cudaStreamCreateWithFlags(&buf.st, cudaStreamNonBlocking));
    TMX_CK(cudaEventCreate(&buf.t0));
    TMX_CK(cudaEventCreate(&buf.t1));
    const int nbuf = precision == TMX_FP16 ? 4 : 2;
    for (int i = 0; i < nbuf; i++) {
        const long long sz = i < 2 ? pbytes : 32 * ps;
        if (cudaMalloc(&buf.p[i], sz) != cudaSuccess) {
            cudaGetLastError();
            return fail(TMX_E_NOMEM, "tmx_pattern_ceiling: no room for %lld bytes", sz);
        }
        TMX_CK(cudaMemsetAsync(buf.p[i], 0, sz, buf.st));
    }
    cudaStream_t st = buf.st;
    cudaEvent_t t0 = buf.t0, t1 = buf.t1;
    // ping-pong between the two buffers, as the interior kernels' A-B pairs
    auto launch = [&](int grid, int r) {
        void* a = buf.p[r & 1];
        void* b = buf.p[(r & 1) ^ 1];
        if (precision == TMX_FP64)
            k_pattern_f64<<<grid, kThreads, 0, st>>>((const double*)a, (double*)b, ps, lo, hi, off, 0);
        else if (precision == TMX_FP32)
            k_pattern_f32<<<grid, kThreads, 0, st>>>((const float4*)a, (float4*)b, ps, lo, hi, off, 0);
        else
            k_pattern_f16<<<grid, kThreads, 0, st>>>((const uint2*)a, (uint2*)b, (const float4*)buf.p[2 + (r & 1)],
                                                     (float4*)buf.p[3 - (r & 1)], ps, lo, hi, off, 0);
    };
    double best = 0.0;
    int best_bps = 0;
    int rc = TMX_OK;
    for (int bps = 1; bps <= 8 && rc == TMX_OK; bps *= 2) {
        const int grid = sms * bps;
        for (int r = 0; r < 3; r++) launch(grid, r);
        cudaEventRecord(t0, st);
        for (int r = 0; r < reps; r++) launch(grid, r);
        cudaEventRecord(t1, st);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (e != cudaSuccess) {
            rc = fail(TMX_E_CUDA, "tmx_pattern_ceiling: %s", cudaGetErrorString(e));
            break;
        }
        const double g = (double)(hi - lo) * bytes_per_node * reps / (ms * 1e-3) / 1e9;
        if (g > best) {
            best = g;
            best_bps = bps;
        }
    }
    if (rc) return rc;
    *gbs = best;
    if (blocks_per_sm) *blocks_per_sm = best_bps;
    return TMX_OK;
}
