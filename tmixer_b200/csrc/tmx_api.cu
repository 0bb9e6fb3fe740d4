// tmx_api.cu -- host side of the C ABI declared in include/tmx.h.
//
// Owns the device state of one T-mixer solve: two population buffers (A-B
// pull), two density buffers (previous / current step, read by boundary
// closures), the macroscopic fields of the last step, the compact boundary
// node list and the inlet profiles.  Kernels are in tmx_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tmx.h"
#include "tmx_classes.h"
#include "tmx_host.h"
#include "tmx_kernels.cuh"

using tmx::Geom;
using tmx::Phys;
using namespace tmx_host;

namespace tmx_host {

thread_local std::string g_err;

const char* last_error() { return g_err.c_str(); }

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

}  // namespace tmx_host

struct tmx_handle {
    tmx_case c;
    Geom G;
    Phys P;
    int device = 0;
    cudaStream_t stream = nullptr;
    // populations (storage type of the form) and densities (its arithmetic type)
    void* pop[2] = {nullptr, nullptr};
    void* rho[2] = {nullptr, nullptr};
    double* mac = nullptr;
    int* bnode = nullptr;
    unsigned char* bcls = nullptr;
    int nb = 0;
    void* uin_d[2] = {nullptr, nullptr};
    float4* mom[2] = {nullptr, nullptr};  // FP16 form: moments of the nodes that wrote pop[s]
    double* stats = nullptr;
    double* partial = nullptr;
    double* diag = nullptr;  // pressure / power outputs (allocated on first use)
    std::vector<double> uin1, uin2;
    std::vector<int> class_count;
    int cur = 0;   // population buffer holding the state
    int rcur = 0;  // density buffer holding the previous step's densities
    long long steps = 0;
    bool inited = false;
    long long bytes = 0;
    int bulk_blocks = 0;
    // the boundary kernel runs on a second stream, concurrently with the bulk
    // kernel (disjoint outputs, read-only shared inputs)
    cudaStream_t aux = nullptr, aux2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr;
    int nface = 0;  // the first nface boundary nodes are face classes
    int nwall = 0;  // the last nwall are wall faces (StepKernels::walls)
    // FP32 / FP16 forms: the last nzwall faces are the z wall faces, which
    // the sweep kernels update (boundary_list)
    int nzwall = 0;
    // one captured step per (state buffer, macroscopic output) combination
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int sbytes = 8, tbytes = 8;  // storage / arithmetic bytes per value of the form
    const struct StepKernels* K = nullptr;
    // interior kernel shape (tmx_set_shape): TMX_SHAPE_*, planes per tile,
    // and the sweep kernels' tile list and grid
    int shape = TMX_SHAPE_FLAT, zchunk = 8;
    int4* tiles = nullptr;
    int ntiles = 0, sweep_blocks = 0;
};

const StepKernels tmx_host::kForms[3] = {
    {tmx::k_init_f64, tmx::k_bulk_f64, nullptr, nullptr, tmx::k_bound_f64, tmx::k_walls_f64, 8, 8, false, true},
    {tmx::k_init_f32, tmx::k_bulk_f32, tmx::k_bfaces_f32, tmx::k_bedges_f32, nullptr, nullptr, 4, 4, false, false},
    {tmx::k_init_f16, tmx::k_bulk_f16, tmx::k_bfaces_f16, tmx::k_bedges_f16, nullptr, nullptr, 2, 4, true, false},
};

namespace tmx_host {

// The FP16 form's equilibrium polynomial (tmx_engine.cuh poly_q_rn), in host
// single precision with every operation rounded on its own.
float poly_q_host(int q, float ux, float uy, float uz, float omt)
{
    const int ex = tmx::EX(q), ey = tmx::EY(q), ez = tmx::EZ(q);
    if (q == 0) return omt;
    const float a = ex > 0 ? ux : -ux, b = ey > 0 ? uy : -uy, c = ez > 0 ? uz : -uz;
    const float eu = ex ? (ey ? a + b : (ez ? a + c : a)) : (ey ? (ez ? b + c : b) : c);
    return std::fmaf(eu, std::fmaf(4.5f, eu, 3.0f), omt);
}

// IEEE binary16 bits to float (host side of tmx_populations)
float half_bits_to_float(unsigned short h)
{
    const unsigned sign = (h >> 15) & 1u, exp = (h >> 10) & 31u, man = h & 1023u;
    float v;
    if (exp == 0) v = std::ldexp((float)man, -24);
    else if (exp == 31) v = man ? NAN : INFINITY;
    else v = std::ldexp((float)(man | 1024u), (int)exp - 25);
    return sign ? -v : v;
}

void geometry_of(const tmx_case& c, Geom& G)
{
    G.inx = c.inx;
    G.iny = c.iny;
    G.nz = c.nz;
    G.mnx = c.mnx;
    G.mny = c.mny;
    G.ia = c.ia;
    G.ib = c.ia + c.mnx - 1;
    G.nx[0] = c.inx;
    G.ny[0] = c.iny;
    G.nx[1] = c.mnx;
    G.ny[1] = c.mny;
    G.base[0] = 0;
    G.base[1] = c.inx * c.iny * c.nz;
    G.nnodes = G.base[1] + c.mnx * c.mny * c.nz;
    G.ps = ((long long)G.nnodes + 63) / 64 * 64;
}

void physics_of(const tmx_case& c, Phys& P)
{
    const double taus[4] = {c.tau, c.tau_a, c.tau_b, c.tau_c};
    for (int f = 0; f < 4; f++) {
        P.c1[f] = (1.0 - 1.0 / taus[f]);  // Tmixer.cpp:9677 "(1.0 - 1.0 / tau)"
        P.c2[f] = (1.0 / taus[f]);
    }
    P.rateconst = c.rateconst;
    P.rho_out = c.rho_out;
    for (int s = 0; s < 3; s++)
        for (int n = 0; n < 2; n++) P.cin[s][n] = c.c_in[s][n];
}

long long footprint(const Geom& G, long long nb, int precision)
{
    const StepKernels& K = kForms[precision];
    long long b = 0;
    b += 2LL * 76 * G.ps * K.sbytes;  // populations
    b += 2LL * 4 * G.ps * K.tbytes;   // densities
    if (K.moments) b += 2LL * 2 * G.ps * 16;  // FP16 form: moments
    b += 7LL * G.ps * 8;       // macroscopic fields
    b += nb * 5;               // boundary list
    b += 2LL * (G.iny + 3) * (G.nz + 3) * K.tbytes;
    b += (long long)(G.mny + G.iny) * 9 * 8 + kSumBlocks * 6 * 8;
    return b;
}

long long boundary_count(const Geom& G)
{
    long long n = 0;
    for (int b = 0; b < 2; b++)
        for (int i = 1; i <= G.nx[b]; i++)
            for (int j = 1; j <= G.ny[b]; j++)
                for (int k = 1; k <= G.nz; k++) n += tmx::is_boundary(G, b, i, j, k);
    return n;
}

// Class of a boundary node, following the node sets of the reference's cases
// (Tmixer.cpp:2023-9033).  Returns -1 for a node no case covers.
int classify(const Geom& G, int b, int i, int j, int k)
{
    using namespace tmx;
    const int nz = G.nz;
    const bool zlo = k == 1, zhi = k == nz, zmid = !zlo && !zhi;
    if (b == 0) {
        const int inx = G.inx, iny = G.iny, ia = G.ia, ib = G.ib;
        const bool ylo = j == 1, yhi = j == iny, ymid = !ylo && !yhi;
        if (i == 1 || i == inx) {
            const bool lo = i == 1;
            if (ylo) return zlo ? (lo ? K_CORNER_1 + 6 : K_CORNER_1 + 7) : zhi ? (lo ? K_CORNER_1 + 2 : K_CORNER_1 + 3)
                                                                              : (lo ? K_EDGE_X1_Y1 : K_EDGE_XT_Y1);
            if (yhi) return zlo ? (lo ? K_CORNER_1 + 4 : K_CORNER_1 + 5) : zhi ? (lo ? K_CORNER_1 + 0 : K_CORNER_1 + 1)
                                                                              : (lo ? K_EDGE_X1_YT : K_EDGE_XT_YT);
            return zlo ? (lo ? K_EDGE_X1_Z1 : K_EDGE_XT_Z1) : zhi ? (lo ? K_EDGE_X1_ZTOP : K_EDGE_XT_ZTOP)
                                                                 : (lo ? K_INLET1 : K_INLET2);
        }
        if (yhi) return zlo ? K_EDGE_YT_Z1 : zhi ? K_EDGE_YT_ZT : K_FACE_YT;
        if (ylo) {
            if (i < ia || i > ib) return zlo ? K_EDGE_Y1_Z1 : zhi ? K_EDGE_Y1_ZTOP : K_FACE_Y1;
            if (i == ia) return zlo ? K_CORNER_1 + 15 : zhi ? K_CORNER_1 + 12 : K_JUNC_DD;
            if (i == ib) return zlo ? K_CORNER_1 + 14 : zhi ? K_CORNER_1 + 13 : K_JUNC_CC;
            return zlo ? K_FACE_Z1 : zhi ? K_FACE_ZT : -1;  // opening nodes of Cases 19 / 17
        }
        (void)ymid;
        if (zlo) return K_FACE_Z1;
        if (zhi) return K_FACE_ZT;
        return -1;
    }
    const int mnx = G.mnx;
    const bool xlo = i == 1, xhi = i == mnx;
    if (j == 1) {
        if (xlo) return zlo ? K_CORNER_1 + 8 : zhi ? K_CORNER_1 + 10 : K_MEDGE_AAp;
        if (xhi) return zlo ? K_CORNER_1 + 9 : zhi ? K_CORNER_1 + 11 : K_MEDGE_BBp;
        return zlo ? K_MEDGE_AB : zhi ? K_MEDGE_ApBp : K_OUTLET;
    }
    if (xlo) return zlo ? K_MEDGE_AD : zhi ? K_MEDGE_ApDp : K_FACE_MX1;
    if (xhi) return zlo ? K_MEDGE_BC : zhi ? K_MEDGE_BpCp : K_FACE_MXT;
    if (zlo) return K_FACE_Z1;
    if (zhi) return K_FACE_ZT;
    (void)zmid;
    return -1;
}

// Inlet profiles exactly as GenerateInletVelocity() (Tmixer.cpp:1426-1539)
// computes them: a rectangular-duct series (100 x 100 terms, libm sin/cos,
// the same loop nesting and operation order), scaled to mean umean, then
// shifted one node down in z (Uin1) and, negated, one node up (Uin2), with
// Uin1[.][1] and Uin2[.][nz] zeroed.
void inlet_series(int iny, int nz, std::vector<double>& U1, double& average)
{
    const int W = nz + 3;
    U1.assign((size_t)(iny + 3) * W, 0.0);
    auto at = [W](std::vector<double>& a, int j, int k) -> double& { return a[(size_t)j * W + k]; };
    const double pi = 3.14159265358979323846;
    const double d = ((nz - 1.0) / 2.0);
    const double w = ((iny - 1.0) / 2.0);
    const double AR = (1.0 * w / d);
    const double den_m = 2.0 * AR * d, den_n = 2.0 * d, AR2 = AR * AR;
    // every (j, k) is an independent sum: rows are spread over host threads,
    // each value computed exactly as a single thread would
    auto rows = [&](int j0, int j1) {
        for (int j = j0; j < j1; j++)
            for (int k = 0; k < nz; k++) {
                double nsum = 0;
                for (int n = 1; n <= 100; n++) {
                    double msum = 0;
                    for (int m = 1; m <= 100; m++) {
                        const double N = (1.0 - std::cos(m * pi)) * (1.0 - std::cos(n * pi)) *
                                         std::sin(((m * pi) / den_m) * (j)) * std::sin(((n * pi) / den_n) * (k));
                        const double D = m * n * ((m * m) + (AR2 * n * n));
                        msum += (N / D);
                    }
                    nsum += msum;
                }
                at(U1, j + 1, k + 1) = nsum;
            }
    };
    const int nt = std::max(1, std::min((int)std::thread::hardware_concurrency(), iny));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(rows, iny * t / nt, iny * (t + 1) / nt);
    rows(0, iny / nt);
    for (auto& th : pool) th.join();
    double sum = 0;
    for (int i = 1; i <= iny; i++)
        for (int j = 1; j <= nz; j++) sum += at(U1, i, j);
    average = sum / ((iny) * (nz));
}

void inlet_scale(const tmx_case& c, const std::vector<double>& raw, double average, std::vector<double>& U1,
                 std::vector<double>& U2)
{
    const int iny = c.iny, nz = c.nz, W = nz + 3;
    U1 = raw;
    U2.assign((size_t)(iny + 3) * W, 0.0);
    auto at = [W](std::vector<double>& a, int j, int k) -> double& { return a[(size_t)j * W + k]; };
    for (int i = 1; i <= iny; i++)
        for (int j = 1; j <= nz; j++) at(U1, i, j) = at(U1, i, j) * (c.umean / average);
    for (int j = 0; j < iny; j++)
        for (int k = 0; k < nz; k++) {
            at(U1, j + 1, k) = at(U1, j + 1, k + 1);
            at(U2, j + 1, k + 2) = -at(U1, j + 1, k);
        }
    for (int i = 1; i <= iny; i++) {
        at(U1, i, 1) = 0;
        at(U2, i, nz) = 0;
    }
}

int inlet_series_device(int iny, int nz, cudaStream_t stream, std::vector<double>& raw, double& average)
{
    const size_t n = (size_t)(iny + 3) * (nz + 3);
    double* d = nullptr;
    TMX_CK(cudaMalloc((void**)&d, n * sizeof(double)));
    cudaError_t e = cudaMemsetAsync(d, 0, n * sizeof(double), stream);
    if (e == cudaSuccess) {
        tmx::k_inlet_series<<<std::max(1, std::min((iny * nz + 127) / 128, 1024)), 128, 0, stream>>>(iny, nz, d);
        e = cudaGetLastError();
    }
    raw.assign(n, 0.0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(raw.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    TMX_CK(e);
    const int W = nz + 3;
    double sum = 0;
    for (int i = 1; i <= iny; i++)
        for (int j = 1; j <= nz; j++) sum += raw[(size_t)i * W + j];
    average = sum / ((iny) * (nz));
    return TMX_OK;
}

int inlet_profile_form(const tmx_case& c, cudaStream_t stream, std::vector<double>& U1, std::vector<double>& U2)
{
    if (c.precision == TMX_FP64) {
        inlet_profile(c, U1, U2);
        return TMX_OK;
    }
    std::vector<double> raw;
    double average;
    int rc = inlet_series_device(c.iny, c.nz, stream, raw, average);
    if (rc) return rc;
    inlet_scale(c, raw, average, U1, U2);
    return TMX_OK;
}

void inlet_profile(const tmx_case& c, std::vector<double>& U1, std::vector<double>& U2)
{
    std::vector<double> raw;
    double average;
    inlet_series(c.iny, c.nz, raw, average);
    inlet_scale(c, raw, average, U1, U2);
}

int boundary_list(const Geom& G, std::vector<int>& nodes, std::vector<unsigned char>& cls, int& nface,
                  std::vector<int>* class_count, int* nwall, int* nzwall)
{
    struct Entry {
        int cls, wall, node;
        bool zwall;
    };
    std::vector<Entry> all;
    all.reserve((size_t)boundary_count(G));
    if (class_count) class_count->assign(tmx::K_NCLASSES, 0);
    bool zsep = nzwall != nullptr && nwall == nullptr;
    long long zcount = 0, interior2 = 0;
    for (int b = 0; b < 2; b++)
        for (int i = 1; i <= G.nx[b]; i++)
            for (int j = 1; j <= G.ny[b]; j++) {
                if (G.nz >= 3 && !tmx::is_boundary(G, b, i, j, 2)) interior2++;
                for (int k = 1; k <= G.nz; k++) {
                    if (!tmx::is_boundary(G, b, i, j, k)) continue;
                    const int c = classify(G, b, i, j, k);
                    if (c < 0)
                        return fail(TMX_E_INVALID, "internal: boundary node (%d,%d,%d,%d) has no class", b, i, j, k);
                    const int w = tmx::wall_class(G, b, i, j, k);
                    if (w != (tmx::is_wall_class(c) ? c : -1))
                        return fail(TMX_E_INVALID, "internal: wall class %d of node (%d,%d,%d,%d), class %d", w, b, i,
                                    j, k, c);
                    if (class_count) (*class_count)[c]++;
                    const bool zw = c == tmx::K_FACE_Z1 || c == tmx::K_FACE_ZT;
                    if (zw) {
                        // the interior node of the column the sweep kernels
                        // update this wall node with (sweep_zwall)
                        const int kw = c == tmx::K_FACE_Z1 ? 1 : G.nz, kn = c == tmx::K_FACE_Z1 ? 2 : G.nz - 1;
                        if (k != kw || G.nz < 3 || tmx::is_boundary(G, b, i, j, kn)) zsep = false;
                        zcount++;
                    }
                    all.push_back({c, w, tmx::node_index(G, b, i, j, k), zw});
                }
            }
    // every z wall node above or below an interior node, and every interior
    // node of planes 2 and nz - 1 under or over one
    if (zcount != 2 * interior2) zsep = false;
    if (nzwall && nwall == nullptr && !zsep && interior2 > 0)
        return fail(TMX_E_INVALID, "internal: the z wall faces do not pair with the interior nodes of planes 2 and %d",
                    G.nz - 1);
    // faces first (with zsep the z wall faces last among them), then edges
    // and corners (then, with nwall, the wall faces); by class, then node
    std::vector<std::pair<int, int>> bl;
    bl.reserve(all.size());
    for (const Entry& e : all) {
        const int key = (nwall && e.wall >= 0)
                            ? 512
                            : (tmx::is_face_class(e.cls) ? (zsep && e.zwall ? 128 : 0) : 256) + e.cls;
        bl.emplace_back(key, e.node);
    }
    std::sort(bl.begin(), bl.end());
    nodes.resize(bl.size());
    cls.resize(bl.size());
    nface = 0;
    int nw = 0, nzw = 0;
    for (size_t t = 0; t < bl.size(); t++) {
        nodes[t] = bl[t].second;
        if (bl[t].first == 512) {  // the walls in node order
            int b, i, j, k;
            tmx::decode(G, nodes[t], b, i, j, k);
            cls[t] = (unsigned char)tmx::wall_class(G, b, i, j, k);
            nw++;
        } else {
            cls[t] = (unsigned char)(bl[t].first & 127);
        }
        if (bl[t].first < 256) nface++;
        if (bl[t].first >= 128 && bl[t].first < 256) nzw++;
    }
    if (nwall) *nwall = nw;
    if (nzwall) *nzwall = nzw;
    return TMX_OK;
}

}  // namespace tmx_host

namespace {

void free_all(tmx_handle* h)
{
    for (int s = 0; s < 2; s++) {
        cudaFree(h->pop[s]);
        cudaFree(h->rho[s]);
        cudaFree(h->uin_d[s]);
        cudaFree(h->mom[s]);
        h->pop[s] = h->rho[s] = h->uin_d[s] = nullptr;
        h->mom[s] = nullptr;
    }
    for (int a = 0; a < 2; a++)
        for (int m = 0; m < 2; m++)
            if (h->graph[a][m]) {
                cudaGraphExecDestroy(h->graph[a][m]);
                h->graph[a][m] = nullptr;
            }
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    if (h->join2) cudaEventDestroy(h->join2);
    h->fork = h->join = h->join2 = nullptr;
    if (h->aux) cudaStreamDestroy(h->aux);
    if (h->aux2) cudaStreamDestroy(h->aux2);
    h->aux = h->aux2 = nullptr;
    cudaFree(h->mac);
    cudaFree(h->bnode);
    cudaFree(h->bcls);
    cudaFree(h->stats);
    cudaFree(h->partial);
    cudaFree(h->tiles);
    h->tiles = nullptr;
    cudaFree(h->diag);
    h->diag = nullptr;
    h->mac = h->stats = h->partial = nullptr;
    h->bnode = nullptr;
    h->bcls = nullptr;
    if (h->stream) cudaStreamDestroy(h->stream);
    h->stream = nullptr;
}

// Queue the two kernels of one step from buffer `cur`: the boundary kernel on
// the auxiliary stream, forked from and joined back into the main stream, and
// the bulk kernel on the main stream.  With ev (4 events) each kernel is
// bracketed by its own pair of events.  The state and density buffers flip
// together every step, so one parity index selects both.
int enqueue_step(tmx_handle* h, int cur, int write_macro, cudaEvent_t* ev)
{
    const Geom& G = h->G;
    tmx::StepPtrs X;
    X.pin = h->pop[cur];
    X.pout = h->pop[1 - cur];
    X.rprev = h->rho[cur];
    X.rcur = h->rho[1 - cur];
    X.mac = h->mac;
    X.mprev = h->mom[cur];
    X.mcur = h->mom[1 - cur];
    X.uin1 = h->uin_d[0];
    X.uin2 = h->uin_d[1];
    TMX_CK(cudaEventRecord(h->fork, h->stream));
    TMX_CK(cudaStreamWaitEvent(h->aux, h->fork, 0));
    TMX_CK(cudaStreamWaitEvent(h->aux2, h->fork, 0));
    if (ev) TMX_CK(cudaEventRecord(ev[2], h->aux));
    const int nf = h->nface, nw = h->nwall, ne = h->nb - h->nface - h->nwall;
    const int bt = tmx::kBoundaryThreadsHost, nl = tmx::kBoundaryLanesHost;  // nl threads per node
    if (h->K->serial) {
        // one launch, the edge and corner blocks first: their long per-node
        // chains then run beside the face blocks instead of after them
        // (W=32 FP64 step 198.5 us against 203.4 us as two launches)
        const int eb = (nl * ne + bt - 1) / bt, fb = (nl * nf + bt - 1) / bt;
        if (eb + fb > 0)
            h->K->bound<<<eb + fb, bt, 0, h->aux>>>(X, h->bnode, h->bcls, nf, ne, eb, G, h->P, write_macro);
        if (nw > 0)
            h->K->walls<<<(nw + bt - 1) / bt, bt, 0, h->aux2>>>(X, h->bnode + nf + ne, h->bcls + nf + ne, nw, G, h->P,
                                                                write_macro);
    } else {
        // with a sweep shape the interior kernel updates the z wall faces,
        // the last nzwall of the face range (zwall_node)
        const int nfk = sweep_shape(h->shape) ? nf - h->nzwall : nf;
        if (nfk > 0)
            h->K->faces<<<(nl * nfk + bt - 1) / bt, bt, 0, h->aux>>>(X, h->bnode, h->bcls, nfk, G, h->P, write_macro);
        if (ne > 0)
            h->K->edges<<<(nl * ne + bt - 1) / bt, bt, 0, h->aux2>>>(X, h->bnode + nf, h->bcls + nf, ne, G, h->P,
                                                                     write_macro);
    }
    TMX_CK(cudaEventRecord(h->join2, h->aux2));
    if (ev) {  // the boundary time spans both boundary kernels
        TMX_CK(cudaStreamWaitEvent(h->aux, h->join2, 0));
        TMX_CK(cudaEventRecord(ev[3], h->aux));
    }
    TMX_CK(cudaEventRecord(h->join, h->aux));
    // FP64: the bulk kernel follows the two boundary kernels.  Its blocks and
    // theirs (about 120 registers each) cannot share an SM, so running them
    // side by side only stretched the bulk launch (step 204 us side by side,
    // 202 us in order at W=32).  The reduced-precision boundary kernels (64
    // registers) do overlap the bulk kernel (FP16 step 75 us side by side,
    // 85 us in order).
    // (timed steps, ev given, run the interior kernel after the boundary
    // kernels in every form, so that each event pair times its kernels alone)
    if (h->K->serial || ev) {
        TMX_CK(cudaStreamWaitEvent(h->stream, h->join, 0));
        TMX_CK(cudaStreamWaitEvent(h->stream, h->join2, 0));
    }
    if (ev) TMX_CK(cudaEventRecord(ev[0], h->stream));
    if (const SweepShape* sh = sweep_shape(h->shape))
        sh->single<<<h->sweep_blocks, sh->threads(), sh->smem(), h->stream>>>(X, G, h->P, write_macro, h->tiles,
                                                                             h->ntiles);
    else
        h->K->bulk<<<h->bulk_blocks, 256, 0, h->stream>>>(X, G, h->P, write_macro);
    if (ev) TMX_CK(cudaEventRecord(ev[1], h->stream));
    if (!h->K->serial && !ev) {
        TMX_CK(cudaStreamWaitEvent(h->stream, h->join, 0));
        TMX_CK(cudaStreamWaitEvent(h->stream, h->join2, 0));
    }
    TMX_CK(cudaGetLastError());
    return TMX_OK;
}

int advance(tmx_handle* h)
{
    h->cur = 1 - h->cur;
    h->rcur = h->cur;
    h->steps++;
    return TMX_OK;
}

// One step through a captured graph (built on first use for this parity and
// output flag).
int graph_step(tmx_handle* h, int write_macro)
{
    cudaGraphExec_t& ex = h->graph[h->cur][write_macro];
    if (!ex) {
        cudaGraph_t gr = nullptr;
        TMX_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(h, h->cur, write_macro, nullptr);
        cudaError_t e = cudaStreamEndCapture(h->stream, &gr);
        if (rc) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        TMX_CK(e);
        e = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        TMX_CK(e);
    }
    TMX_CK(cudaGraphLaunch(ex, h->stream));
    return advance(h);
}

int timed_step(tmx_handle* h, int write_macro, cudaEvent_t* ev)
{
    int rc = enqueue_step(h, h->cur, write_macro, ev);
    if (rc) return rc;
    return advance(h);
}

}  // namespace

namespace tmx_host {

int check_case(const tmx_case& cc)
{
    const tmx_case* c = &cc;
    if (c->inx < 3 || c->iny < 3 || c->nz < 3 || c->mnx < 3 || c->mny < 3)
        return fail(TMX_E_INVALID, "every box size must be >= 3 (inx=%d iny=%d nz=%d mnx=%d mny=%d)", c->inx, c->iny,
                    c->nz, c->mnx, c->mny);
    if (c->ia < 2 || c->ia + c->mnx - 1 > c->inx - 1)
        return fail(TMX_E_INVALID, "opening columns ia=%d..ib=%d must lie within 2..inx-1=%d", c->ia,
                    c->ia + c->mnx - 1, c->inx - 1);
    const double t[4] = {c->tau, c->tau_a, c->tau_b, c->tau_c};
    for (double v : t)
        if (!(v > 0.5) || !std::isfinite(v)) return fail(TMX_E_INVALID, "relaxation times must be finite and > 0.5");
    if (!std::isfinite(c->rho0) || !(c->rho0 > 0) || !std::isfinite(c->rho_out) || !(c->rho_out > 0))
        return fail(TMX_E_INVALID, "rho0 and rho_out must be finite and positive");
    if (!std::isfinite(c->umean) || !std::isfinite(c->rateconst)) return fail(TMX_E_INVALID, "non-finite parameter");
    if (c->precision < TMX_FP64 || c->precision > TMX_FP16)
        return fail(TMX_E_INVALID, "unsupported precision %d", c->precision);
    const long long n = (long long)c->inx * c->iny * c->nz + (long long)c->mnx * c->mny * c->nz;
    if (n > 2000000000LL) return fail(TMX_E_INVALID, "too many nodes (%lld)", n);
    return TMX_OK;
}

// Two cases are the same solve: every field equal (the struct's padding
// bytes are not compared, so a case filled member by member matches one
// cleared with memset first).  Doubles compare by their bits.
static bool same_case(const tmx_case& a, const tmx_case& b)
{
    auto same = [](double x, double y) { return std::memcmp(&x, &y, sizeof x) == 0; };
    bool eq = a.inx == b.inx && a.iny == b.iny && a.nz == b.nz && a.mnx == b.mnx && a.mny == b.mny && a.ia == b.ia &&
              a.precision == b.precision && same(a.tau, b.tau) && same(a.tau_a, b.tau_a) && same(a.tau_b, b.tau_b) &&
              same(a.tau_c, b.tau_c) && same(a.rho0, b.rho0) && same(a.rho_out, b.rho_out) &&
              same(a.rateconst, b.rateconst) && same(a.umean, b.umean);
    for (int s = 0; s < 3; s++)
        for (int n = 0; n < 2; n++) eq = eq && same(a.c_in[s][n], b.c_in[s][n]);
    return eq;
}

int checkpoint_check(const void* buf, long long size, const tmx_case& c, const Geom& G)
{
    if (size < (long long)sizeof(CheckpointHeader)) return fail(TMX_E_INVALID, "checkpoint too small");
    CheckpointHeader hd;
    std::memcpy(&hd, buf, sizeof hd);
    if (std::memcmp(hd.magic, "TMXCKPT1", 8) == 0)
        return fail(TMX_E_INVALID, "checkpoint of an earlier format (FP16 moment records ordered differently)");
    if (std::memcmp(hd.magic, kCheckpointMagic, 8) != 0) return fail(TMX_E_INVALID, "not a checkpoint");
    if (hd.abi != TMX_ABI_VERSION) return fail(TMX_E_INVALID, "checkpoint of ABI %d, library %d", hd.abi, TMX_ABI_VERSION);
    if (hd.precision != c.precision)
        return fail(TMX_E_INVALID, "checkpoint of precision %d, target %d", hd.precision, c.precision);
    if (!same_case(hd.c, c)) return fail(TMX_E_INVALID, "checkpoint of a different case");
    long long b[5];
    checkpoint_sections(G, c.precision, b);
    if (hd.ps != G.ps || std::memcmp(hd.bytes, b, sizeof b) != 0 || size != checkpoint_total(b))
        return fail(TMX_E_INVALID, "checkpoint sizes do not match the case");
    if (hd.steps < 0) return fail(TMX_E_INVALID, "checkpoint with a negative step count");
    return TMX_OK;
}

}  // namespace tmx_host

extern "C" {

int tmx_abi_version(void) { return TMX_ABI_VERSION; }

const char* tmx_last_error(void) { return last_error(); }

int tmx_case_reference(tmx_case* out)
{
    if (!out) return fail(TMX_E_INVALID, "tmx_case_reference: null output");
    std::memset(out, 0, sizeof *out);
    out->inx = 401;
    out->iny = 51;
    out->nz = 51;
    out->mnx = 101;
    out->mny = 800 - 50;
    out->ia = ((401 + 1) / 2) - ((101 - 1) / 2);
    out->tau = 0.6;
    const double tc = (0.5 * (((2.0 * 0.6 - 1.0) / 3.0) + 1.0));
    out->tau_a = out->tau_b = out->tau_c = tc;
    out->rho0 = 3.0;
    out->rho_out = 3.0;
    out->c_in[0][0] = 1.0;
    out->c_in[1][1] = 1.0;
    out->rateconst = 1.0;
    out->umean = 0.059761;
    out->precision = TMX_FP64;
    return TMX_OK;
}

int tmx_case_wlayout(int W, double u_max, double tau_f, double tau_c, double k, double rho, tmx_case* out)
{
    if (!out) return fail(TMX_E_INVALID, "tmx_case_wlayout: null output");
    if (W < 3) return fail(TMX_E_INVALID, "tmx_case_wlayout: W=%d must be >= 3", W);
    if (!(u_max > 0) || !std::isfinite(u_max)) return fail(TMX_E_INVALID, "u_max must be positive");
    tmx_case c;
    std::memset(&c, 0, sizeof c);
    c.inx = 8 * W;
    c.iny = W;
    c.nz = W;
    c.mnx = 2 * W;
    c.mny = 4 * W;
    c.ia = 3 * W + 1;
    c.tau = tau_f;
    c.tau_a = c.tau_b = c.tau_c = tau_c;
    c.rho0 = rho;
    c.rho_out = rho;
    c.c_in[0][0] = 1.0;
    c.c_in[1][1] = 1.0;
    c.rateconst = k;
    c.umean = 1.0;
    c.precision = TMX_FP64;
    std::vector<double> U1, U2;
    inlet_profile(c, U1, U2);
    double mx = 0.0;
    for (double v : U1) mx = std::max(mx, v);
    if (!(mx > 0)) return fail(TMX_E_INVALID, "degenerate inlet profile");
    c.umean = u_max / mx;
    *out = c;
    return tmx_case_check(out);
}

int tmx_case_check(const tmx_case* c)
{
    if (!c) return fail(TMX_E_INVALID, "null case");
    return check_case(*c);
}


int tmx_case_footprint(const tmx_case* c, long long* bytes)
{
    int rc = tmx_case_check(c);
    if (rc) return rc;
    if (!bytes) return fail(TMX_E_INVALID, "null output");
    Geom G;
    geometry_of(*c, G);
    *bytes = footprint(G, boundary_count(G), c->precision);
    return TMX_OK;
}

int tmx_create(const tmx_case* c, int device, tmx_handle** out)
{
    if (!out) return fail(TMX_E_INVALID, "null output handle");
    *out = nullptr;
    int rc = tmx_case_check(c);
    if (rc) return rc;
    int ndev = 0;
    TMX_CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(TMX_E_INVALID, "device %d out of range (%d devices)", device, ndev);
    TMX_CK(cudaSetDevice(device));

    tmx_handle* h = new tmx_handle();
    h->c = *c;
    h->device = device;
    geometry_of(*c, h->G);
    physics_of(*c, h->P);
    h->K = &kForms[c->precision];
    h->sbytes = h->K->sbytes;
    h->tbytes = h->K->tbytes;
    const Geom& G = h->G;

    // boundary node list, faces first, sorted by class then node index
    std::vector<int> nodes;
    std::vector<unsigned char> cls;
    rc = boundary_list(G, nodes, cls, h->nface, &h->class_count, h->K->walls ? &h->nwall : nullptr, &h->nzwall);
    if (rc) {
        delete h;
        return rc;
    }
    h->nb = (int)nodes.size();

    auto alloc = [&](void** p, size_t n) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, n);
        if (e == cudaSuccess) h->bytes += (long long)n;
        return e;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->aux2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join2, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
    for (int s = 0; s < 2 && e == cudaSuccess; s++) {
        e = alloc((void**)&h->pop[s], (size_t)76 * G.ps * h->sbytes);
        if (e == cudaSuccess) e = alloc((void**)&h->rho[s], (size_t)4 * G.ps * h->tbytes);
        if (e == cudaSuccess) e = alloc((void**)&h->uin_d[s], (size_t)(G.iny + 3) * (G.nz + 3) * h->tbytes);
        if (e == cudaSuccess && h->K->moments) e = alloc((void**)&h->mom[s], (size_t)2 * G.ps * sizeof(float4));
    }
    if (e == cudaSuccess) e = alloc((void**)&h->mac, (size_t)7 * G.ps * sizeof(double));
    if (e == cudaSuccess) e = alloc((void**)&h->bnode, std::max<size_t>(1, nodes.size()) * sizeof(int));
    if (e == cudaSuccess) e = alloc((void**)&h->bcls, std::max<size_t>(1, cls.size()));
    if (e == cudaSuccess) e = alloc((void**)&h->stats, (size_t)(G.mny + G.iny) * 9 * sizeof(double));
    if (e == cudaSuccess) e = alloc((void**)&h->partial, (size_t)kSumBlocks * 6 * sizeof(double));
    if (e == cudaSuccess && h->nb)
        e = cudaMemcpy(h->bnode, nodes.data(), nodes.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h->nb) e = cudaMemcpy(h->bcls, cls.data(), cls.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? TMX_E_NOMEM : TMX_E_CUDA;
        free_all(h);
        delete h;
        cudaGetLastError();
        return fail(code, "tmx_create: %s", cudaGetErrorString(e));
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    h->bulk_blocks = std::max(1, std::min((G.nnodes + 255) / 256, sms * 8));
    // the FP16 form's interior as 32 x 4 sweep tiles of 8 planes (the same
    // bits as the flat kernel, faster: W=32 step 61 us against 69 us)
    if (h->K->moments) {
        const int rc = tmx_set_shape(h, TMX_SHAPE_SWEEP4, 8);
        if (rc) {
            const std::string msg = last_error();
            tmx_destroy(h);
            return fail(rc, "%s", msg.c_str());
        }
    }
    *out = h;
    return TMX_OK;
}

int tmx_set_shape(tmx_handle* h, int kind, int zchunk)
{
    if (!h) return fail(TMX_E_INVALID, "null handle");
    const SweepShape* sh = sweep_shape(kind);
    if (kind != TMX_SHAPE_FLAT && !sh) return fail(TMX_E_INVALID, "tmx_set_shape: unknown kind %d", kind);
    if (sh && !h->K->moments)
        return fail(TMX_E_INVALID, "tmx_set_shape: the sweep shapes are for the FP16 form only");
    if (sh && zchunk < 1) return fail(TMX_E_INVALID, "tmx_set_shape: zchunk must be >= 1");
    TMX_CK(cudaSetDevice(h->device));
    TMX_CK(cudaStreamSynchronize(h->stream));
    if (sh) {
        TMX_CK(sweep_allow_smem());
        std::vector<int4> t;
        sweep_tiles(h->G, 0, sh->ty, zchunk, t);
        int4* d = nullptr;
        if (!t.empty()) {
            cudaError_t e = cudaMalloc((void**)&d, t.size() * sizeof(int4));
            if (e == cudaSuccess) e = cudaMemcpy(d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(d);
                cudaGetLastError();
                return fail(e == cudaErrorMemoryAllocation ? TMX_E_NOMEM : TMX_E_CUDA, "tmx_set_shape: %s",
                            cudaGetErrorString(e));
            }
        }
        int per = 1, sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)sh->single, sh->threads(), sh->smem());
        cudaGetLastError();
        cudaFree(h->tiles);
        h->tiles = d;
        h->ntiles = (int)t.size();
        h->sweep_blocks = std::max(1, std::min(h->ntiles, sms * std::max(1, per)));
    }
    h->shape = kind;
    h->zchunk = zchunk;
    for (auto& row : h->graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    return TMX_OK;
}

int tmx_init(tmx_handle* h)
{
    if (!h) return fail(TMX_E_INVALID, "null handle");
    TMX_CK(cudaSetDevice(h->device));
    int rc = inlet_profile_form(h->c, h->stream, h->uin1, h->uin2);
    if (rc) return rc;
    if (h->tbytes == 8) {
        const size_t nu = h->uin1.size() * sizeof(double);
        TMX_CK(cudaMemcpy(h->uin_d[0], h->uin1.data(), nu, cudaMemcpyHostToDevice));
        TMX_CK(cudaMemcpy(h->uin_d[1], h->uin2.data(), nu, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> a(h->uin1.begin(), h->uin1.end()), b(h->uin2.begin(), h->uin2.end());
        TMX_CK(cudaMemcpy(h->uin_d[0], a.data(), a.size() * sizeof(float), cudaMemcpyHostToDevice));
        TMX_CK(cudaMemcpy(h->uin_d[1], b.data(), b.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    h->cur = 0;
    h->rcur = 0;
    tmx::StepPtrs X{};
    X.pout = h->pop[0];
    X.rcur = h->rho[0];
    X.mac = h->mac;
    X.mcur = h->mom[0];
    h->K->init<<<h->bulk_blocks, 256, 0, h->stream>>>(X, h->G, h->P, h->c.rho0);
    TMX_CK(cudaGetLastError());
    TMX_CK(cudaStreamSynchronize(h->stream));
    h->steps = 0;
    h->inited = true;
    return TMX_OK;
}

int tmx_step(tmx_handle* h, int nsteps)
{
    if (!h) return fail(TMX_E_INVALID, "null handle");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_step before tmx_init");
    if (nsteps < 0) return fail(TMX_E_INVALID, "negative step count");
    TMX_CK(cudaSetDevice(h->device));
    for (int s = 0; s < nsteps; s++) {
        int rc = graph_step(h, s == nsteps - 1);
        if (rc) return rc;
    }
    return TMX_OK;
}

int tmx_sync(tmx_handle* h)
{
    if (!h) return fail(TMX_E_INVALID, "null handle");
    TMX_CK(cudaSetDevice(h->device));
    TMX_CK(cudaStreamSynchronize(h->stream));
    return TMX_OK;
}

long long tmx_steps_done(const tmx_handle* h) { return h ? h->steps : -1; }

int tmx_checkpoint_size(const tmx_handle* h, long long* bytes)
{
    if (!h || !bytes) return fail(TMX_E_INVALID, "null argument");
    long long b[5];
    checkpoint_sections(h->G, h->c.precision, b);
    *bytes = checkpoint_total(b);
    return TMX_OK;
}

int tmx_checkpoint(tmx_handle* h, void* buf, long long size)
{
    if (!h || !buf) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_checkpoint before tmx_init");
    long long b[5];
    checkpoint_sections(h->G, h->c.precision, b);
    if (size != checkpoint_total(b)) return fail(TMX_E_INVALID, "checkpoint buffer of %lld bytes, %lld needed", size,
                                                 checkpoint_total(b));
    TMX_CK(cudaSetDevice(h->device));
    TMX_CK(cudaStreamSynchronize(h->stream));
    CheckpointHeader hd{};
    std::memcpy(hd.magic, kCheckpointMagic, 8);
    hd.abi = TMX_ABI_VERSION;
    hd.precision = h->c.precision;
    hd.c = h->c;
    hd.steps = h->steps;
    hd.ps = h->G.ps;
    std::memcpy(hd.bytes, b, sizeof b);
    char* p = (char*)buf;
    std::memcpy(p, &hd, sizeof hd);
    p += sizeof hd;
    const void* src[4] = {h->pop[h->cur], h->rho[h->cur], h->mom[h->cur], h->mac};
    for (int k = 0; k < 4; k++) {
        if (b[k]) TMX_CK(cudaMemcpy(p, src[k], (size_t)b[k], cudaMemcpyDeviceToHost));
        p += b[k];
    }
    std::memcpy(p, h->uin1.data(), (size_t)b[4] / 2);
    std::memcpy(p + b[4] / 2, h->uin2.data(), (size_t)b[4] / 2);
    return TMX_OK;
}

int tmx_restore(tmx_handle* h, const void* buf, long long size)
{
    if (!h || !buf) return fail(TMX_E_INVALID, "null argument");
    int rc = checkpoint_check(buf, size, h->c, h->G);
    if (rc) return rc;
    TMX_CK(cudaSetDevice(h->device));
    TMX_CK(cudaStreamSynchronize(h->stream));
    CheckpointHeader hd;
    std::memcpy(&hd, buf, sizeof hd);
    const char* p = (const char*)buf + sizeof hd;
    // the state goes into buffer set 0, which the next step then reads
    void* dst[4] = {h->pop[0], h->rho[0], h->mom[0], h->mac};
    for (int k = 0; k < 4; k++) {
        if (hd.bytes[k]) TMX_CK(cudaMemcpy(dst[k], p, (size_t)hd.bytes[k], cudaMemcpyHostToDevice));
        p += hd.bytes[k];
    }
    const size_t nu = (size_t)(h->G.iny + 3) * (h->G.nz + 3);
    h->uin1.assign((const double*)p, (const double*)p + nu);
    h->uin2.assign((const double*)p + nu, (const double*)p + 2 * nu);
    if (h->tbytes == 8) {
        TMX_CK(cudaMemcpy(h->uin_d[0], h->uin1.data(), nu * 8, cudaMemcpyHostToDevice));
        TMX_CK(cudaMemcpy(h->uin_d[1], h->uin2.data(), nu * 8, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> a(h->uin1.begin(), h->uin1.end()), c(h->uin2.begin(), h->uin2.end());
        TMX_CK(cudaMemcpy(h->uin_d[0], a.data(), nu * 4, cudaMemcpyHostToDevice));
        TMX_CK(cudaMemcpy(h->uin_d[1], c.data(), nu * 4, cudaMemcpyHostToDevice));
    }
    h->cur = 0;
    h->rcur = 0;
    h->steps = hd.steps;
    h->inited = true;
    return TMX_OK;
}

int tmx_case_of(const tmx_handle* h, tmx_case* out)
{
    if (!h || !out) return fail(TMX_E_INVALID, "null argument");
    *out = h->c;
    return TMX_OK;
}

// Copy n = nx*ny*nz doubles of one box from the device (x fastest) into host
// memory in the reference's [i][j][k] order (k fastest).
static int box_to_host(tmx_handle* h, int box, const double* dev, double* host_out, std::vector<double>& stage)
{
    const Geom& G = h->G;
    const int nx = G.nx[box], ny = G.ny[box], nz = G.nz;
    const size_t n = (size_t)nx * ny * nz;
    stage.resize(n);
    TMX_CK(cudaMemcpyAsync(stage.data(), dev + G.base[box], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TMX_CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++) {
            const double* src = stage.data() + ((size_t)k * ny + j) * nx;
            for (int i = 0; i < nx; i++) host_out[((size_t)i * ny + j) * nz + k] = src[i];
        }
    return TMX_OK;
}

int tmx_fields(tmx_handle* h, int box, int field, double* host_out)
{
    if (!h || !host_out) return fail(TMX_E_INVALID, "null argument");
    if (box < 0 || box > 1 || field < 0 || field > 6) return fail(TMX_E_INVALID, "box %d / field %d out of range", box, field);
    if (!h->inited) return fail(TMX_E_STATE, "tmx_fields before tmx_init");
    TMX_CK(cudaSetDevice(h->device));
    std::vector<double> stage;
    return box_to_host(h, box, h->mac + (size_t)field * h->G.ps, host_out, stage);
}

int tmx_populations(tmx_handle* h, int box, int fld, double* host_out)
{
    if (!h || !host_out) return fail(TMX_E_INVALID, "null argument");
    if (box < 0 || box > 1 || fld < 0 || fld > 3) return fail(TMX_E_INVALID, "box %d / field %d out of range", box, fld);
    if (!h->inited) return fail(TMX_E_STATE, "tmx_populations before tmx_init");
    TMX_CK(cudaSetDevice(h->device));
    const Geom& G = h->G;
    const size_t n = (size_t)G.nx[box] * G.ny[box] * G.nz;
    std::vector<double> stage;
    if (h->sbytes == 8) {
        for (int q = 0; q < 19; q++) {
            const double* src = (const double*)h->pop[h->cur] + (size_t)(fld * 19 + q) * G.ps;
            int rc = box_to_host(h, box, src, host_out + q * n, stage);
            if (rc) return rc;
        }
        return TMX_OK;
    }
    // reduced precision: widen on the host; the FP16 form adds back feq of
    // the writing node's moments exactly as the kernels do (tmx_engine.cuh)
    std::vector<double> wide(n);
    std::vector<unsigned char> raw(4 * n * h->sbytes);
    // moment records {(rho, cA, cB, cC), (ux, uy, uz, 1 - 1.5|u|^2)}, 8 floats per node
    std::vector<float> mr(8 * n);
    if (h->K->moments) {
        const float4* m = h->mom[h->cur];
        TMX_CK(cudaMemcpy(mr.data(), m + 2 * (size_t)G.base[box], n * 2 * sizeof(float4), cudaMemcpyDeviceToHost));
    }
    for (int q = 0; q < 19; q++) {
        // interleaved layout: the four fields of (q, node) side by side
        const unsigned char* src =
            (const unsigned char*)h->pop[h->cur] + ((size_t)q * G.ps + G.base[box]) * 4 * h->sbytes;
        TMX_CK(cudaMemcpy(raw.data(), src, raw.size(), cudaMemcpyDeviceToHost));
        const float w = (float)(q == 0 ? 1.0 / 3.0 : (q <= 6 ? 1.0 / 18.0 : 1.0 / 36.0));
        for (size_t t = 0; t < n; t++) {
            float v;
            const size_t e = (t * 4 + fld) * h->sbytes;
            if (h->sbytes == 4) {
                std::memcpy(&v, &raw[e], 4);
            } else {
                unsigned short hb;
                std::memcpy(&hb, &raw[e], 2);
                const float* rec = &mr[8 * t];
                const float r = rec[fld];
                const float pw = poly_q_host(q, rec[4], rec[5], rec[6], rec[7]) * w;
                v = std::fmaf(r, pw, half_bits_to_float(hb));
            }
            wide[t] = v;
        }
        const int nx = G.nx[box], ny = G.ny[box], nz = G.nz;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++)
                    host_out[q * n + ((size_t)i * ny + j) * nz + k] = wide[((size_t)k * ny + j) * nx + i];
    }
    return TMX_OK;
}

int tmx_mixing(tmx_handle* h, double* rows_out, double* outlet_im)
{
    if (!h || !rows_out) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_mixing before tmx_init");
    TMX_CK(cudaSetDevice(h->device));
    const Geom& G = h->G;
    const int nrow = G.mny + G.iny;
    tmx::k_mixing_rows<<<nrow, 32, 0, h->stream>>>(h->mac, G, h->stats);
    TMX_CK(cudaGetLastError());
    std::vector<double> st((size_t)nrow * 9);
    TMX_CK(cudaMemcpyAsync(st.data(), h->stats, st.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TMX_CK(cudaStreamSynchronize(h->stream));
    // running maxima over the rows in the reference's order, starting at 0
    double mx[3] = {0.0, 0.0, 0.0};
    for (int r = 0; r < nrow; r++) {
        const double* s = &st[(size_t)r * 9];
        double* o = rows_out + (size_t)r * 7;
        const bool mixing_row = r < G.mny;
        o[0] = mixing_row ? r + 1 : (r - G.mny + 1) + G.mny;
        for (int q = 0; q < 3; q++) {
            if (mx[q] < s[6 + q]) mx[q] = s[6 + q];
            o[1 + q] = s[q];
        }
        const bool ok = mixing_row ? (s[0] > 0 && s[1] > 0 && s[2] > 0) : (s[0] > 0);
        for (int q = 0; q < 3; q++) {
            if (ok) {
                const double Is = s[3 + q] / (s[q] * (mx[q] - s[q]));
                o[4 + q] = 1.0 - std::sqrt(Is);
            } else {
                o[4 + q] = 0.0;
            }
        }
    }
    if (outlet_im)
        for (int q = 0; q < 3; q++) outlet_im[q] = rows_out[4 + q];
    return TMX_OK;
}

// Scratch address of tmx_mixing_static per device, resolved by the first
// call on that device (cudaGetSymbolAddress with the device current).
namespace {
constexpr int kMixStaticDevices = 64;
std::once_flag g_mix_once[kMixStaticDevices];
double* g_mix_ptr[kMixStaticDevices];
cudaError_t g_mix_err[kMixStaticDevices];
}  // namespace

int tmx_mixing_static(tmx_handle* h, double* rows_out, double* outlet_im)
{
    if (!h || !rows_out) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_mixing_static before tmx_init");
    const Geom& G = h->G;
    const int nrow = G.mny + G.iny;
    if (nrow > tmx::kMixStaticRows)
        return fail(TMX_E_INVALID,
                    "tmx_mixing_static: mny + iny = %d rows exceeds its fixed scratch of %d rows (use tmx_mixing)",
                    nrow, tmx::kMixStaticRows);
    const int d = h->device;
    if (d < 0 || d >= kMixStaticDevices)
        return fail(TMX_E_INVALID, "tmx_mixing_static: device %d is beyond its table of %d devices", d,
                    kMixStaticDevices);
    TMX_CK(cudaSetDevice(d));
    std::call_once(g_mix_once[d], [d] { g_mix_err[d] = tmx::mixing_static_scratch(&g_mix_ptr[d]); });
    if (g_mix_err[d] != cudaSuccess)
        return fail(TMX_E_CUDA, "tmx_mixing_static: cudaGetSymbolAddress on device %d: %s", d,
                    cudaGetErrorString(g_mix_err[d]));
    double* stats = g_mix_ptr[d];
    double* rows = stats + (size_t)tmx::kMixStaticRows * 9;
    tmx::k_mixing_rows<<<nrow, 32, 0, h->stream>>>(h->mac, G, stats);
    tmx::k_mixing_finish<<<1, 96, 0, h->stream>>>(stats, G, rows);
    TMX_CK(cudaGetLastError());
    TMX_CK(cudaMemcpyAsync(rows_out, rows, (size_t)nrow * 7 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TMX_CK(cudaStreamSynchronize(h->stream));
    if (outlet_im)
        for (int q = 0; q < 3; q++) outlet_im[q] = rows_out[4 + q];
    return TMX_OK;
}

int tmx_sums(tmx_handle* h, double out[8])
{
    if (!h || !out) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_sums before tmx_init");
    TMX_CK(cudaSetDevice(h->device));
    tmx::k_sums<<<kSumBlocks, 256, 0, h->stream>>>(h->mac, h->G, h->partial);
    TMX_CK(cudaGetLastError());
    std::vector<double> p((size_t)kSumBlocks * 6);
    TMX_CK(cudaMemcpyAsync(p.data(), h->partial, p.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TMX_CK(cudaStreamSynchronize(h->stream));
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < kSumBlocks; b++)
        for (int m = 0; m < 6; m++) s[m] += p[(size_t)b * 6 + m];
    out[0] = s[0];
    out[1] = s[1];
    out[2] = s[2];
    out[3] = s[3];
    out[4] = s[1] + s[2] + s[3];
    out[5] = s[4];
    out[6] = s[5];
    out[7] = (double)h->G.nnodes;
    return TMX_OK;
}

int tmx_pressure_power(tmx_handle* h, double* pressure_rows, double* pressure_x, double* power_rows,
                       double units[2])
{
    if (!h || !pressure_rows || !pressure_x || !power_rows || !units) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_pressure_power before tmx_init");
    TMX_CK(cudaSetDevice(h->device));
    const Geom& G = h->G;
    const int nrow = G.mny + G.iny, npow = G.mny - 2, nout = 1 + nrow + G.inx + 4 * npow;
    if (!h->diag) {
        cudaError_t e = cudaMalloc((void**)&h->diag, (size_t)nout * sizeof(double));
        if (e != cudaSuccess) {
            h->diag = nullptr;
            cudaGetLastError();
            return fail(e == cudaErrorMemoryAllocation ? TMX_E_NOMEM : TMX_E_CUDA, "tmx_pressure_power: %s",
                        cudaGetErrorString(e));
        }
        h->bytes += (long long)nout * sizeof(double);
    }
    const int items = 1 + nrow + G.inx + npow;
    tmx::k_pressure_power<<<(items + 127) / 128, 128, 0, h->stream>>>(h->mac, G, h->c.tau, h->diag);
    TMX_CK(cudaGetLastError());
    std::vector<double> o((size_t)nout);
    TMX_CK(cudaMemcpyAsync(o.data(), h->diag, o.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TMX_CK(cudaStreamSynchronize(h->stream));
    const double ptop = o[0];
    for (int r = 0; r < nrow; r++) {
        pressure_rows[3 * r] = r + 1;  // mixing rows 1..mny, then inlet row j as j + mny
        pressure_rows[3 * r + 1] = o[1 + r];
        pressure_rows[3 * r + 2] = o[1 + r] - ptop;
    }
    for (int i = 0; i < G.inx; i++) {
        pressure_x[2 * i] = i + 1;
        pressure_x[2 * i + 1] = o[1 + nrow + i];
    }
    for (int j = 0; j < npow; j++) {
        power_rows[5 * j] = j + 2;
        for (int m = 0; m < 4; m++) power_rows[5 * j + 1 + m] = o[1 + nrow + G.inx + 4 * j + m];
    }
    // the reference's unit factors (Tmixer.cpp:185-196: LENGTH 0.0008 m, PRESSURE
    // 101325 Pa, KVISCOSITY 1.004e-6 m^2/s, length = inx), as its macros expand
    const double tau = h->c.tau, rho0 = h->c.rho0;
    const double L0 = (0.0008 / (G.inx - 1));
    const double T0 = ((((2.0 * tau - 1.0) / 6.0) / 0.000001004) * (L0 * L0));
    const double M0 = ((101325.0 / (rho0 / 3.0)) * (L0 * T0 * T0));
    units[0] = ((M0) / (L0 * T0 * T0));
    units[1] = ((L0 * L0) / (T0 * T0 * T0));
    return TMX_OK;
}

int tmx_inlet_profile(tmx_handle* h, double* uin1, double* uin2)
{
    if (!h || !uin1 || !uin2) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_inlet_profile before tmx_init");
    std::memcpy(uin1, h->uin1.data(), h->uin1.size() * sizeof(double));
    std::memcpy(uin2, h->uin2.data(), h->uin2.size() * sizeof(double));
    return TMX_OK;
}

int tmx_step_timed(tmx_handle* h, int nsteps, double* ms_bulk, double* ms_boundary, double* ms_total)
{
    if (!h) return fail(TMX_E_INVALID, "null handle");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_step_timed before tmx_init");
    if (nsteps <= 0) return fail(TMX_E_INVALID, "nsteps must be positive");
    TMX_CK(cudaSetDevice(h->device));
    std::vector<cudaEvent_t> ev((size_t)nsteps * 4);
    for (auto& x : ev) TMX_CK(cudaEventCreate(&x));
    cudaEvent_t t0, t1;
    TMX_CK(cudaEventCreate(&t0));
    TMX_CK(cudaEventCreate(&t1));
    TMX_CK(cudaEventRecord(t0, h->stream));
    int rc = TMX_OK;
    for (int s = 0; s < nsteps && rc == TMX_OK; s++) rc = timed_step(h, s == nsteps - 1, &ev[(size_t)s * 4]);
    TMX_CK(cudaEventRecord(t1, h->stream));
    TMX_CK(cudaEventSynchronize(t1));
    double sb = 0, sbd = 0;
    for (int s = 0; s < nsteps && rc == TMX_OK; s++) {
        float a = 0, b = 0;
        TMX_CK(cudaEventElapsedTime(&a, ev[(size_t)s * 4], ev[(size_t)s * 4 + 1]));
        TMX_CK(cudaEventElapsedTime(&b, ev[(size_t)s * 4 + 2], ev[(size_t)s * 4 + 3]));
        sb += a;
        sbd += b;
    }
    float tot = 0;
    TMX_CK(cudaEventElapsedTime(&tot, t0, t1));
    for (auto& x : ev) cudaEventDestroy(x);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    if (ms_bulk) *ms_bulk = sb;
    if (ms_boundary) *ms_boundary = sbd;
    if (ms_total) *ms_total = tot;
    return TMX_OK;
}

int tmx_time_steps(tmx_handle* h, int nsteps, double* ms)
{
    if (!h || !ms) return fail(TMX_E_INVALID, "null argument");
    if (!h->inited) return fail(TMX_E_STATE, "tmx_time_steps before tmx_init");
    if (nsteps <= 0) return fail(TMX_E_INVALID, "nsteps must be positive");
    TMX_CK(cudaSetDevice(h->device));
    cudaEvent_t t0, t1;
    TMX_CK(cudaEventCreate(&t0));
    TMX_CK(cudaEventCreate(&t1));
    TMX_CK(cudaEventRecord(t0, h->stream));
    int rc = tmx_step(h, nsteps);
    TMX_CK(cudaEventRecord(t1, h->stream));
    TMX_CK(cudaEventSynchronize(t1));
    float el = 0;
    TMX_CK(cudaEventElapsedTime(&el, t0, t1));
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    *ms = el;
    return TMX_OK;
}

int tmx_counts(const tmx_handle* h, long long out[4])
{
    if (!h || !out) return fail(TMX_E_INVALID, "null argument");
    out[0] = h->G.nnodes;
    out[1] = h->G.nnodes - h->nb;
    out[2] = h->nb;
    out[3] = h->bytes;
    return TMX_OK;
}

void tmx_destroy(tmx_handle* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
}

}  // extern "C"
