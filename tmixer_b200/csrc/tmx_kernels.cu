// tmx_kernels.cu -- sm_100a kernels of the plain FP64 form (bit-exact with
// the reference) and the FP64 reductions over the macroscopic fields.  This
// translation unit is compiled with --fmad=false: every multiply and add is
// rounded separately, as in the reference's x86-64 build; the only fused
// operations are the explicit __fma_rn of the correctly rounded constant
// divisions (tmx_device.cuh).  The step itself is in tmx_engine.cuh.
#include "tmx_engine.cuh"

namespace tmx {

TMX_DEFINE_STEP_KERNELS(F64, f64)
TMX_DEFINE_BOUND_KERNEL(F64, f64)
TMX_DEFINE_WALL_KERNEL(F64, f64)
TMX_DEFINE_BATCH_KERNELS(F64, f64)

// ---------------------------------------------------------------------------
// mixing quality (Tmixer.cpp:10161-10409): per row, per species, the sums of
// the reference in its order (k inner, i outer), then per-row maxima.  One
// thread block per row; thread s handles species s.  Rows: mixing 1..mny,
// then inlet 1..iny over x = ia..ib.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void row_stats(const double* __restrict__ Mac, const Geom& G, int row, int s, double& avg,
                                          double& var, double& mx)
{
    const int b = row < G.mny ? 1 : 0;
    const int j = b == 1 ? row + 1 : row - G.mny + 1;
    const int i0 = b == 1 ? 1 : G.ia, i1 = b == 1 ? G.mnx : G.ib;
    const double* cfield = Mac + (long long)(4 + s) * G.ps;
    double sumx = 0.0;
    mx = __longlong_as_double(0xfff0000000000000ULL);  // -inf
    for (int i = i0; i <= i1; i++) {
        double sumz = 0.0;
        for (int k = 1; k <= G.nz; k++) {
            const double v = cfield[node_index(G, b, i, j, k)];
            sumz += v;
            mx = fmax(mx, v);
        }
        sumx += sumz;
    }
    avg = (sumx / (1.0 * G.nz * G.mnx));
    sumx = 0.0;
    for (int i = i0; i <= i1; i++) {
        double sumz = 0.0;
        for (int k = 1; k <= G.nz; k++) {
            const double d = cfield[node_index(G, b, i, j, k)] - avg;
            sumz += d * d;
        }
        sumx += sumz;
    }
    var = (1.0 / (1.0 * G.nz * G.mnx)) * sumx;
}

__global__ void k_mixing_rows(const double* __restrict__ Mac, Geom G, double* __restrict__ stats)
{
    const int row = blockIdx.x;
    const int s = threadIdx.x;
    if (s >= 3) return;
    double avg, var, mx;
    row_stats(Mac, G, row, s, avg, var, mx);
    stats[row * 9 + s] = avg;
    stats[row * 9 + 3 + s] = var;
    stats[row * 9 + 6 + s] = mx;
}

// Outlet row (mixing row 1, the first row of the reference's order) of batch
// mixers: its running maximum is max(0, the row's maximum).  One block per
// entry, thread s handles species s.
__global__ void k_outlet_im_batch(const MixerDesc* __restrict__ D, const int* __restrict__ slots, int n,
                                  double* __restrict__ out)
{
    const int e = blockIdx.x, s = threadIdx.x;
    __shared__ double avgs[3];
    if (e >= n) return;
    const MixerDesc& d = D[slots[e]];
    double avg = 0.0, var = 0.0, m = 0.0;
    if (s < 3) {
        row_stats(d.X[0].mac, d.G, 0, s, avg, var, m);
        avgs[s] = avg;
    }
    __syncthreads();
    if (s >= 3) return;
    double mx = 0.0;
    if (mx < m) mx = m;
    const bool ok = avgs[0] > 0 && avgs[1] > 0 && avgs[2] > 0;
    out[3 * e + s] = ok ? 1.0 - sqrt(var / (avg * (mx - avg))) : 0.0;
}

__global__ void k_nonfinite_batch(const MixerDesc* __restrict__ D, const int4* __restrict__ blocks,
                                  const int* __restrict__ counts, int* __restrict__ flags)
{
    const int nblk = counts[0];
    for (int b = blockIdx.x; b < nblk; b += gridDim.x) {
        const int4 cb = blocks[b];
        const MixerDesc& d = D[cb.x];
        const double* mac = d.X[0].mac;
        const long long ps = d.G.ps;
        bool bad = false;
        for (int t = threadIdx.x; t < cb.z; t += blockDim.x)
            for (int f = 0; f < 7; f++) bad |= !isfinite(mac[f * ps + cb.y + t]);
        if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&flags[cb.x], 1);
    }
}

// ---------------------------------------------------------------------------
// The rectangular-duct series of GenerateInletVelocity (Tmixer.cpp:1426-1480)
// on the device, for the reduced-precision forms: raw[(j+1)*(nz+3) + k+1] =
// sum over m, n = 1..100 of (1 - cos m pi)(1 - cos n pi) sin(m pi j / (2 AR d))
// sin(n pi k / (2 d)) / (m n (m^2 + AR^2 n^2)), j < iny, k < nz.  The factors
// (1 - cos m pi) are exactly 0 for even m and 2 for odd m, so only odd m and n
// are summed, with sinpi for the sines.  Agrees with the host's libm series to
// about 1e-15 relative (the FP64 form keeps the host series, bit for bit).
// ---------------------------------------------------------------------------
__global__ void k_inlet_series(int iny, int nz, double* __restrict__ raw)
{
    const double d = ((nz - 1.0) / 2.0), w = ((iny - 1.0) / 2.0);
    const double AR = (1.0 * w / d), AR2 = AR * AR;
    const double den_m = 2.0 * AR * d, den_n = 2.0 * d;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < iny * nz; t += gridDim.x * blockDim.x) {
        const int j = t / nz, k = t % nz;
        double nsum = 0.0;
        for (int n = 1; n <= 100; n += 2) {
            const double sn = sinpi((n * (double)k) / den_n);
            double msum = 0.0;
            for (int m = 1; m <= 100; m += 2) {
                const double N = 4.0 * sinpi((m * (double)j) / den_m) * sn;
                const double D = (double)(m * n) * ((double)(m * m) + (AR2 * n * n));
                msum += N / D;
            }
            nsum += msum;
        }
        raw[(j + 1) * (nz + 3) + (k + 1)] = nsum;
    }
}

// ---------------------------------------------------------------------------
// Fixed device scratch of tmx_mixing_static (no allocation in that call).
// Every word the call reads is written earlier in the same call, so nothing
// in it has to start at zero.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_mix_scratch[kMixStaticRows * (9 + 7)];

cudaError_t mixing_static_scratch(double** ptr) { return cudaGetSymbolAddress((void**)ptr, g_mix_scratch); }

// Finish the rows of write_MixingQuality() (Tmixer.cpp:10161-10409) on the
// device, with the same arithmetic as the host finish of tmx_mixing: running
// maxima over the rows in the reference's order starting at 0, then
// I_s = 1 - sqrt(var / (avg * (max - avg))).  One warp per species; lane l
// takes a contiguous chunk of rows, and a shuffle scan of the chunk maxima
// gives each chunk its running maximum on entry.  The update "if (m < v)
// m = v" from 0 keeps m = max(+0, non-NaN values), whatever the grouping, so
// the chunked scan equals the sequential one bit for bit.
__global__ void k_mixing_finish(const double* __restrict__ stats, Geom G, double* __restrict__ rows)
{
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q >= 3) return;
    const int nrow = G.mny + G.iny;
    const int chunk = (nrow + 31) / 32;
    const int r0 = min(lane * chunk, nrow), r1 = min(r0 + chunk, nrow);
    double m = 0.0;
    for (int r = r0; r < r1; r++) {
        const double v = stats[r * 9 + 6 + q];
        if (m < v) m = v;
    }
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, m, o);
        if (lane >= o && m < y) m = y;
    }
    double mx = __shfl_up_sync(0xffffffffu, m, 1);
    if (lane == 0) mx = 0.0;
    for (int r = r0; r < r1; r++) {
        const double* s = stats + r * 9;
        double* o = rows + r * 7;
        const bool mixing_row = r < G.mny;
        if (q == 0) o[0] = mixing_row ? r + 1 : (r - G.mny + 1) + G.mny;
        if (mx < s[6 + q]) mx = s[6 + q];
        o[1 + q] = s[q];
        const bool ok = mixing_row ? (s[0] > 0 && s[1] > 0 && s[2] > 0) : (s[0] > 0);
        o[4 + q] = ok ? 1.0 - sqrt(s[3 + q] / (s[q] * (mx - s[q]))) : 0.0;
    }
}

// ---------------------------------------------------------------------------
// Pressure and specific power (the numbers of write_Pressure_Power,
// Tmixer.cpp:9866-10027), one thread per output item, each a sequential sum
// in the reference's order.  out: [0] the pressure of inlet row iny over the
// opening (p_top), [1 .. nrow] the row pressures (mixing rows 1..mny, inlet
// rows 1..iny over x = ia..ib), then inx cross-section pressures of the inlet
// box, then for each mixing row j = 2..mny-1 four rates: cross-section and
// total as the reference computes them (its x loop assigns rather than adds,
// so only column mnx-1 enters the sums over k) and the same two summed over
// every column.  Pressures are mean density / 3; rates use
// vis = (2 tau - 1) / 6 and the central differences of the velocity.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mean_row_rho(const double* __restrict__ rho, const Geom& G, int b, int j, int i0,
                                               int i1)
{
    double sumx = 0.0;
    for (int i = i0; i <= i1; i++) {
        double sumz = 0.0;
        for (int k = 1; k <= G.nz; k++) sumz += rho[node_index(G, b, i, j, k)];
        sumx += sumz;
    }
    return (sumx / (1.0 * G.nz * G.mnx)) / 3.0;
}

__global__ void k_pressure_power(const double* __restrict__ Mac, Geom G, double tau, double* __restrict__ out)
{
    const int nrow = G.mny + G.iny, nitems = 1 + nrow + G.inx + (G.mny - 2);
    const double* rho = Mac;
    const double *ux = Mac + G.ps, *uy = Mac + 2 * G.ps, *uz = Mac + 3 * G.ps;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nitems; t += gridDim.x * blockDim.x) {
        if (t == 0) {
            out[0] = mean_row_rho(rho, G, 0, G.iny, G.ia, G.ib);
        } else if (t <= nrow) {
            const int r = t - 1;
            out[t] = r < G.mny ? mean_row_rho(rho, G, 1, r + 1, 1, G.mnx)
                               : mean_row_rho(rho, G, 0, r - G.mny + 1, G.ia, G.ib);
        } else if (t <= nrow + G.inx) {
            const int i = t - nrow;
            double sumy = 0.0;
            for (int j = 1; j <= G.iny; j++) {
                double sumz = 0.0;
                for (int k = 1; k <= G.nz; k++) sumz += rho[node_index(G, 0, i, j, k)];
                sumy += sumz;
            }
            out[t] = (sumy / (1.0 * G.nz * G.iny)) / 3.0;
        } else {
            const int j = t - nrow - G.inx + 1;  // 2 .. mny-1
            const double vis = ((2.0 * tau - 1.0) / 6.0) * (1.0 * 1.0 * 1.0);
            double sumz = 0.0, sumtotalz = 0.0, allz = 0.0, alltotalz = 0.0;
            for (int k = 2; k < G.nz; k++) {
                double sx = 0.0, stx = 0.0, allx = 0.0, alltx = 0.0;
                for (int i = 2; i < G.mnx; i++) {
#define TMX_M(a, ii, jj, kk) a[node_index(G, 1, ii, jj, kk)]
                    const double delux = (TMX_M(ux, i + 1, j, k) - TMX_M(ux, i - 1, j, k)) / 2.0;
                    const double delvy = (TMX_M(uy, i, j + 1, k) - TMX_M(uy, i, j - 1, k)) / 2.0;
                    const double delwz = (TMX_M(uz, i, j, k + 1) - TMX_M(uz, i, j, k - 1)) / 2.0;
                    const double deluy = (TMX_M(ux, i, j + 1, k) - TMX_M(ux, i, j - 1, k)) / 2.0;
                    const double delvx = (TMX_M(uy, i + 1, j, k) - TMX_M(uy, i - 1, j, k)) / 2.0;
                    const double deluz = (TMX_M(ux, i, j, k + 1) - TMX_M(ux, i, j, k - 1)) / 2.0;
                    const double delwx = (TMX_M(uz, i + 1, j, k) - TMX_M(uz, i - 1, j, k)) / 2.0;
                    const double delvz = (TMX_M(uy, i, j, k + 1) - TMX_M(uy, i, j, k - 1)) / 2.0;
                    const double delwy = (TMX_M(uz, i, j + 1, k) - TMX_M(uz, i, j - 1, k)) / 2.0;
#undef TMX_M
                    const double a = deluz + delwx, bxy = delvx + deluy, c = delvz + delwy;
                    sx = delux * delux + delwz * delwz + 0.5 * (a * a);
                    stx = delux * delux + delvy * delvy + delwz * delwz + 0.5 * (bxy * bxy) + 0.5 * (a * a) +
                          0.5 * (c * c);
                    allx += sx;
                    alltx += stx;
                }
                sumz += sx;
                sumtotalz += stx;
                allz += allx;
                alltotalz += alltx;
            }
            const double n = 1.0 * (G.nz - 2) * (G.mnx - 2);
            double* o = out + 1 + nrow + G.inx + 4 * (j - 2);
            o[0] = 2.0 * vis * (sumz / n);
            o[1] = 2.0 * vis * (sumtotalz / n);
            o[2] = 2.0 * vis * (allz / n);
            o[3] = 2.0 * vis * (alltotalz / n);
        }
    }
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
