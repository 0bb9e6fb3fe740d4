// tmx_batch.cu -- the batched engine behind tmx_batch_* (include/tmx.h): many
// T-mixers of uneven size and parameters stepped together, every step one
// launch per kernel kind over all of them.
//
//   - Device memory: one arena of the batch's budget, allocated once; each
//     mixer's state is a first-fit range of it (admission by footprint).
//   - Work lists: the bulk kernel walks a concatenated list of cell blocks
//     {mixer, first node, node count}; the boundary kernels walk the
//     concatenated face and edge node lists {node, mixer * 256 + class}.  A
//     mixer's descriptor (buffers per step parity, geometry, physics) is
//     read from device memory; the sweep and boundary kernels copy it into
//     shared memory once per tile or per 32 list entries (the lists are
//     padded so that those belong to one mixer).
//   - Step parity: a batch-wide counter; a mixer admitted when the counter's
//     parity is p reads its initial buffer at parity p (the descriptor's two
//     buffer sets are swapped accordingly), so mixers of different ages step
//     together.
//   - The lists, descriptors and counts live in device memory at fixed
//     addresses, so the captured step graphs stay valid while mixers come and
//     go; they are recaptured only when a list outgrows its capacity or the
//     tuned launch shape changes.
//   - tmx_batch_tune times each interior-kernel shape on the batch's own
//     mixers and keeps the fastest: the flat kernel's block size and
//     cell-block size, and (FP16 form) the sweep kernels' tile height and
//     planes per tile, i.e. nodes per thread.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/tmx.h"
#include "tmx_classes.h"
#include "tmx_host.h"
#include "tmx_kernels.cuh"

using tmx::Geom;
using tmx::MixerDesc;
using tmx::Phys;
using namespace tmx_host;

namespace {

using BulkBatchFn = void (*)(const MixerDesc*, const int4*, const int*, int, int);
using BoundaryBatchFn = void (*)(const MixerDesc*, const int2*, const int*, int, int);

struct BatchKernels {
    BulkBatchFn bulk[3];  // 128, 256, 512 threads per block
    BoundaryBatchFn faces, edges;
};
const BatchKernels kBatchForms[3] = {
    {{tmx::k_bulk_batch128_f64, tmx::k_bulk_batch256_f64, tmx::k_bulk_batch512_f64}, tmx::k_bfaces_batch_f64,
     tmx::k_bedges_batch_f64},
    {{tmx::k_bulk_batch128_f32, tmx::k_bulk_batch256_f32, tmx::k_bulk_batch512_f32}, tmx::k_bfaces_batch_f32,
     tmx::k_bedges_batch_f32},
    {{tmx::k_bulk_batch128_f16, tmx::k_bulk_batch256_f16, tmx::k_bulk_batch512_f16}, tmx::k_bfaces_batch_f16,
     tmx::k_bedges_batch_f16},
};
constexpr int kBulkThreads[3] = {128, 256, 512};
constexpr int kCellChoices[4] = {1024, 2048, 4096, 8192};
constexpr long long kAlign = 256;

long long align_up(long long x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Device bytes of one batch mixer, in the order its buffers are carved.
struct Carve {
    long long pop, rho, uin, mom, mac, total;
};
Carve carve_of(const Geom& G, int precision)
{
    const StepKernels& K = kForms[precision];
    Carve c;
    c.pop = align_up(76LL * G.ps * K.sbytes);
    c.rho = align_up(4LL * G.ps * K.tbytes);
    c.uin = align_up((long long)(G.iny + 3) * (G.nz + 3) * K.tbytes);
    c.mom = K.moments ? align_up(2LL * G.ps * 16) : 0;
    c.mac = align_up(7LL * G.ps * 8);
    c.total = 2 * (c.pop + c.rho + c.uin + c.mom) + c.mac;
    return c;
}

struct Slot {
    bool used = false;
    tmx_case c{};
    Geom G{};
    Phys P{};
    long long off = 0, bytes = 0;  // arena range
    void* pop[2] = {nullptr, nullptr};
    void* rho[2] = {nullptr, nullptr};
    void* uin[2] = {nullptr, nullptr};
    float4* mom[2] = {nullptr, nullptr};
    double* mac = nullptr;
    std::vector<int> nodes;
    std::vector<unsigned char> cls;
    int nface = 0;
    int nzwall = 0;  // z wall faces last among the faces (boundary_list)
    int parity0 = 0;  // batch parity at admission
    long long steps = 0;
};

// First-fit allocator over [0, capacity) with coalescing frees.
struct Arena {
    long long capacity = 0;
    std::map<long long, long long> free_;  // offset -> size
    void reset(long long cap)
    {
        capacity = cap;
        free_.clear();
        if (cap > 0) free_[0] = cap;
    }
    long long alloc(long long n)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                const long long off = it->first, left = it->second - n;
                free_.erase(it);
                if (left > 0) free_[off + n] = left;
                return off;
            }
        return -1;
    }
    void release(long long off, long long n)
    {
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    long long free_bytes() const
    {
        long long s = 0;
        for (auto& kv : free_) s += kv.second;
        return s;
    }
    long long largest() const
    {
        long long s = 0;
        for (auto& kv : free_) s = std::max(s, kv.second);
        return s;
    }
};

// The duct series depends on (iny, nz) only: computed once per shape.
std::mutex g_series_mu;
std::map<std::pair<int, int>, std::pair<std::vector<double>, double>> g_series;

// (one cache per arithmetic: the host series for FP64, the device series for
// the reduced-precision forms)
int cached_inlet(const tmx_case& c, cudaStream_t stream, std::vector<double>& U1, std::vector<double>& U2)
{
    const bool host = c.precision == TMX_FP64;
    std::pair<std::vector<double>, double> e;
    {
        std::lock_guard<std::mutex> lk(g_series_mu);
        auto it = g_series.find({host ? c.iny : -c.iny, c.nz});
        if (it != g_series.end()) e = it->second;
    }
    if (e.first.empty()) {
        if (host) {
            inlet_series(c.iny, c.nz, e.first, e.second);
        } else {
            int rc = inlet_series_device(c.iny, c.nz, stream, e.first, e.second);
            if (rc) return rc;
        }
        std::lock_guard<std::mutex> lk(g_series_mu);
        g_series[{host ? c.iny : -c.iny, c.nz}] = e;
    }
    inlet_scale(c, e.first, e.second, U1, U2);
    return TMX_OK;
}

}  // namespace

struct tmx_batch {
    int device = 0;
    int precision = TMX_FP16;
    const StepKernels* K = nullptr;
    const BatchKernels* B = nullptr;
    cudaStream_t stream = nullptr, aux = nullptr, aux2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, join2 = nullptr;
    char* arena_base = nullptr;
    Arena arena;
    std::vector<Slot> slots;
    // device tables (fixed addresses between reallocations)
    MixerDesc* d_desc = nullptr;
    int cap_desc = 0;
    int4* d_blocks = nullptr;
    int cap_blocks = 0;
    int4* d_tiles = nullptr;  // sweep kernel tiles (FP16 form)
    int cap_tiles = 0;
    int2* d_faces = nullptr;
    int cap_faces = 0;
    int2* d_edges = nullptr;
    int cap_edges = 0;
    int* d_counts = nullptr;
    int* d_slots = nullptr;
    double* d_im = nullptr;
    int* d_flags = nullptr;  // per-slot health flags (tmx_batch_health)
    int cap_flags = 0;
    int cap_im = 0;
    long long table_bytes = 0;
    bool dirty = true;
    int parity = 0;
    long long steps = 0;
    // launch shape
    int variant = 1;     // index into kBulkThreads
    int cells = 4096;    // nodes per cell block
    int sweep = 0;       // 0: the flat kernel; else the TMX_SHAPE_SWEEP* shape of the interior
    int zchunk = 8;      // planes per sweep tile
    int bound_bps = 0;   // boundary kernels' blocks per SM (0: as many as fit)
    int bound_after = 0; // reduced-precision forms: interior kernel after the boundary kernels (1) or beside them
    int bound_fit = 1;   // blocks of the face kernel that fit on an SM
    int sms = 148;
    int grid_bulk[3] = {0, 0, 0};
    int grid_sweep[4] = {0, 0, 0, 0};  // by TMX_SHAPE_SWEEP* kind
    int grid_faces = 0, grid_edges = 0;
    int nblocks = 0, nfaces = 0, nedges = 0, ntiles = 0, nactive = 0;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
};

namespace {

void drop_graphs(tmx_batch* b)
{
    for (auto& row : b->graph)
        for (auto& g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
}

template <class E>
cudaError_t grow(tmx_batch* b, E*& ptr, int& cap, int need)
{
    if (need <= cap) return cudaSuccess;
    int n = std::max(need, std::max(64, cap * 2));
    if (ptr) {
        cudaStreamSynchronize(b->stream);
        cudaFree(ptr);
        b->table_bytes -= (long long)cap * sizeof(E);
        ptr = nullptr;
        cap = 0;
    }
    drop_graphs(b);
    cudaError_t e = cudaMalloc((void**)&ptr, (size_t)n * sizeof(E));
    if (e == cudaSuccess) {
        cap = n;
        b->table_bytes += (long long)n * sizeof(E);
    }
    return e;
}

MixerDesc desc_of(const tmx_batch* b, const Slot& s)
{
    MixerDesc d{};
    d.G = s.G;
    d.P = s.P;
    for (int p = 0; p < 2; p++) {
        // at batch parity p the mixer has taken (p - parity0) mod 2 steps, so
        // its state is in buffer q = (p ^ parity0)
        const int q = p ^ s.parity0;
        tmx::StepPtrs& X = d.X[p];
        X.pin = s.pop[q];
        X.pout = s.pop[1 - q];
        X.rprev = s.rho[q];
        X.rcur = s.rho[1 - q];
        X.mac = s.mac;
        X.mprev = s.mom[q];
        X.mcur = s.mom[1 - q];
        X.uin1 = s.uin[0];
        X.uin2 = s.uin[1];
    }
    (void)b;
    return d;
}

// Rebuild descriptors and work lists of the used slots and upload them.
int rebuild(tmx_batch* b)
{
    std::vector<MixerDesc> desc(b->slots.size());
    std::vector<int4> blocks, tiles;
    std::vector<int2> faces, edges;
    int nactive = 0;
    for (size_t m = 0; m < b->slots.size(); m++) {
        const Slot& s = b->slots[m];
        if (!s.used) continue;
        nactive++;
        desc[m] = desc_of(b, s);
        for (int g0 = 0; g0 < s.G.nnodes; g0 += b->cells)
            blocks.push_back(make_int4((int)m, g0, std::min(b->cells, s.G.nnodes - g0), 0));
        if (b->sweep) sweep_tiles(s.G, (int)m, sweep_shape(b->sweep)->ty, b->zchunk, tiles);
        // with a sweep shape the interior kernel updates the z wall faces,
        // the last nzwall of the face range (zwall_node)
        const int nfk = b->sweep ? s.nface - s.nzwall : s.nface;
        for (size_t t = 0; t < s.nodes.size(); t++) {
            const int2 e = make_int2(s.nodes[t], (int)m * 256 + s.cls[t]);
            if ((int)t < s.nface) {
                if ((int)t < nfk) faces.push_back(e);
            } else {
                edges.push_back(e);
            }
        }
        // each mixer's entries start at a multiple of kListAlign, so that
        // the kListAlign entries a block takes at a time belong to one mixer
        const int2 pad = make_int2(-1, (int)m * 256);
        while (faces.size() % tmx::kListAlign) faces.push_back(pad);
        while (edges.size() % tmx::kListAlign) edges.push_back(pad);
    }
    cudaError_t e = grow(b, b->d_desc, b->cap_desc, (int)std::max<size_t>(1, desc.size()));
    if (e == cudaSuccess) e = grow(b, b->d_blocks, b->cap_blocks, (int)std::max<size_t>(1, blocks.size()));
    if (e == cudaSuccess) e = grow(b, b->d_faces, b->cap_faces, (int)std::max<size_t>(1, faces.size()));
    if (e == cudaSuccess) e = grow(b, b->d_edges, b->cap_edges, (int)std::max<size_t>(1, edges.size()));
    if (e == cudaSuccess) e = grow(b, b->d_tiles, b->cap_tiles, (int)std::max<size_t>(1, tiles.size()));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? TMX_E_NOMEM : TMX_E_CUDA, "batch tables: %s",
                    cudaGetErrorString(e));
    }
    // stream-ordered uploads (pageable sources are staged before the calls
    // return); no step of the old lists is in flight (callers synchronise
    // before changing slots)
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    if (!desc.empty()) TMX_CK(cudaMemcpyAsync(b->d_desc, desc.data(), desc.size() * sizeof(MixerDesc), h2d, b->stream));
    if (!blocks.empty())
        TMX_CK(cudaMemcpyAsync(b->d_blocks, blocks.data(), blocks.size() * sizeof(int4), h2d, b->stream));
    if (!faces.empty()) TMX_CK(cudaMemcpyAsync(b->d_faces, faces.data(), faces.size() * sizeof(int2), h2d, b->stream));
    if (!edges.empty()) TMX_CK(cudaMemcpyAsync(b->d_edges, edges.data(), edges.size() * sizeof(int2), h2d, b->stream));
    if (!tiles.empty()) TMX_CK(cudaMemcpyAsync(b->d_tiles, tiles.data(), tiles.size() * sizeof(int4), h2d, b->stream));
    const int counts[4] = {(int)blocks.size(), (int)faces.size(), (int)edges.size(), (int)tiles.size()};
    TMX_CK(cudaMemcpyAsync(b->d_counts, counts, sizeof counts, h2d, b->stream));
    TMX_CK(cudaStreamSynchronize(b->stream));
    b->nblocks = counts[0];
    b->nfaces = counts[1];
    b->nedges = counts[2];
    b->ntiles = counts[3];
    b->nactive = nactive;
    b->dirty = false;
    return TMX_OK;
}

// One batch step on the batch's streams.  With ev (4 events: interior start
// and end, boundary start and end) the interior kernel runs after the
// boundary kernels in every form, so that each event pair times its kernels
// alone (tmx_batch_step_timed).
int enqueue(tmx_batch* b, int parity, int write_macro, cudaEvent_t* ev = nullptr)
{
    TMX_CK(cudaEventRecord(b->fork, b->stream));
    TMX_CK(cudaStreamWaitEvent(b->aux, b->fork, 0));
    TMX_CK(cudaStreamWaitEvent(b->aux2, b->fork, 0));
    if (ev) TMX_CK(cudaEventRecord(ev[2], b->aux));
    const int bt = tmx::kBoundaryThreadsHost;
    b->B->faces<<<b->grid_faces, bt, 0, b->aux>>>(b->d_desc, b->d_faces, b->d_counts, parity, write_macro);
    b->B->edges<<<b->grid_edges, bt, 0, b->aux2>>>(b->d_desc, b->d_edges, b->d_counts, parity, write_macro);
    TMX_CK(cudaEventRecord(b->join2, b->aux2));
    if (ev) {
        TMX_CK(cudaStreamWaitEvent(b->aux, b->join2, 0));
        TMX_CK(cudaEventRecord(ev[3], b->aux));
    }
    TMX_CK(cudaEventRecord(b->join, b->aux));
    // in order for FP64, side by side for the reduced-precision forms (as the
    // single-mixer step; StepKernels::serial)
    if (b->K->serial || b->bound_after || ev) {
        TMX_CK(cudaStreamWaitEvent(b->stream, b->join, 0));
        TMX_CK(cudaStreamWaitEvent(b->stream, b->join2, 0));
    }
    if (ev) TMX_CK(cudaEventRecord(ev[0], b->stream));
    if (const SweepShape* sh = b->sweep ? sweep_shape(b->sweep) : nullptr)
        sh->batch<<<b->grid_sweep[b->sweep], sh->threads(), sh->smem(), b->stream>>>(b->d_desc, b->d_tiles,
                                                                                    b->d_counts, parity, write_macro);
    else
        b->B->bulk[b->variant]<<<b->grid_bulk[b->variant], kBulkThreads[b->variant], 0, b->stream>>>(
            b->d_desc, b->d_blocks, b->d_counts, parity, write_macro);
    TMX_CK(cudaGetLastError());
    if (ev) TMX_CK(cudaEventRecord(ev[1], b->stream));
    if (!b->K->serial && !b->bound_after && !ev) {
        TMX_CK(cudaStreamWaitEvent(b->stream, b->join, 0));
        TMX_CK(cudaStreamWaitEvent(b->stream, b->join2, 0));
    }
    return TMX_OK;
}

int step_one(tmx_batch* b, int write_macro)
{
    const int p = b->parity;
    cudaGraphExec_t& ge = b->graph[p][write_macro];
    if (!ge) {
        cudaGraph_t g = nullptr;
        cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
        TMX_CK(cudaStreamBeginCapture(b->stream, mode));
        int rc = enqueue(b, p, write_macro);
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        TMX_CK(e);
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        TMX_CK(e);
    }
    TMX_CK(cudaGraphLaunch(ge, b->stream));
    b->parity ^= 1;
    b->steps++;
    return TMX_OK;
}

void set_grids(tmx_batch* b)
{
    for (int v = 0; v < 3; v++) {
        int per = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)b->B->bulk[v], kBulkThreads[v], 0);
        b->grid_bulk[v] = b->sms * std::max(1, per);
    }
    if (b->K->moments && sweep_allow_smem() == cudaSuccess)
        for (int kind = TMX_SHAPE_SWEEP8; kind <= TMX_SHAPE_SWEEP4; kind++) {
            const SweepShape* sh = sweep_shape(kind);
            int per = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)sh->batch, sh->threads(), sh->smem());
            b->grid_sweep[kind] = b->sms * std::max(1, per);
        }
    int pf = 1, pe = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf, (const void*)b->B->faces, tmx::kBoundaryThreadsHost, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pe, (const void*)b->B->edges, tmx::kBoundaryThreadsHost, 0);
    pf = std::max(1, pf);
    pe = std::max(1, pe);
    b->bound_fit = pf;
    // persistent boundary grids: bound_bps blocks per SM, or as many as fit
    b->grid_faces = b->sms * (b->bound_bps > 0 ? std::min(b->bound_bps, pf) : pf);
    b->grid_edges = b->sms * (b->bound_bps > 0 ? std::min(b->bound_bps, pe) : pe);
    cudaGetLastError();
}

int init_slot(tmx_batch* b, Slot& s)
{
    std::vector<double> u1, u2;
    int rc = cached_inlet(s.c, b->stream, u1, u2);
    if (rc) return rc;
    if (b->K->tbytes == 8) {
        TMX_CK(cudaMemcpyAsync(s.uin[0], u1.data(), u1.size() * 8, cudaMemcpyHostToDevice, b->stream));
        TMX_CK(cudaMemcpyAsync(s.uin[1], u2.data(), u2.size() * 8, cudaMemcpyHostToDevice, b->stream));
    } else {
        std::vector<float> a(u1.begin(), u1.end()), c(u2.begin(), u2.end());
        TMX_CK(cudaMemcpyAsync(s.uin[0], a.data(), a.size() * 4, cudaMemcpyHostToDevice, b->stream));
        TMX_CK(cudaMemcpyAsync(s.uin[1], c.data(), c.size() * 4, cudaMemcpyHostToDevice, b->stream));
    }
    tmx::StepPtrs X{};
    X.pout = s.pop[0];
    X.rcur = s.rho[0];
    X.mac = s.mac;
    X.mcur = s.mom[0];
    const int blocks = std::max(1, std::min((s.G.nnodes + 255) / 256, b->sms * 8));
    b->K->init<<<blocks, 256, 0, b->stream>>>(X, s.G, s.P, s.c.rho0);
    TMX_CK(cudaGetLastError());
    s.parity0 = b->parity;
    s.steps = 0;
    return TMX_OK;
}

bool valid_slot(const tmx_batch* b, int slot) { return slot >= 0 && slot < (int)b->slots.size() && b->slots[slot].used; }

}  // namespace

extern "C" {

int tmx_batch_footprint(const tmx_case* c, long long* bytes)
{
    if (!c || !bytes) return fail(TMX_E_INVALID, "null argument");
    int rc = check_case(*c);
    if (rc) return rc;
    Geom G;
    geometry_of(*c, G);
    *bytes = carve_of(G, c->precision).total;
    return TMX_OK;
}

int tmx_batch_create(int precision, long long budget_bytes, int device, tmx_batch** out)
{
    if (!out) return fail(TMX_E_INVALID, "null output");
    *out = nullptr;
    if (precision < TMX_FP64 || precision > TMX_FP16) return fail(TMX_E_INVALID, "unsupported precision %d", precision);
    if (budget_bytes <= 0) return fail(TMX_E_INVALID, "budget must be positive");
    int ndev = 0;
    TMX_CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(TMX_E_INVALID, "device %d out of range (%d devices)", device, ndev);
    TMX_CK(cudaSetDevice(device));
    tmx_batch* b = new tmx_batch();
    b->device = device;
    b->precision = precision;
    b->K = &kForms[precision];
    b->B = &kBatchForms[precision];
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    const long long budget = align_up(budget_bytes);
    cudaError_t e = cudaMalloc((void**)&b->arena_base, (size_t)budget);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->aux2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join2, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_counts, 4 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_counts, 0, 4 * sizeof(int));
    if (e != cudaSuccess) {
        cudaGetLastError();
        tmx_batch_destroy(b);
        return fail(e == cudaErrorMemoryAllocation ? TMX_E_NOMEM : TMX_E_CUDA, "tmx_batch_create: %s",
                    cudaGetErrorString(e));
    }
    b->arena.reset(budget);
    set_grids(b);
    *out = b;
    return TMX_OK;
}

}  // extern "C"

namespace {

// Restore a checkpoint (format in tmx_host.h) into a freshly carved slot: the
// state goes into buffer set 0 with parity0 = the batch's parity, so the
// next batch step reads it.
int restore_slot(tmx_batch* b, Slot& s, const void* buf, long long size)
{
    int rc = checkpoint_check(buf, size, s.c, s.G);
    if (rc) return rc;
    CheckpointHeader hd;
    std::memcpy(&hd, buf, sizeof hd);
    const char* p = (const char*)buf + sizeof hd;
    void* dst[4] = {s.pop[0], s.rho[0], s.mom[0], s.mac};
    for (int k = 0; k < 4; k++) {
        if (hd.bytes[k]) TMX_CK(cudaMemcpyAsync(dst[k], p, (size_t)hd.bytes[k], cudaMemcpyHostToDevice, b->stream));
        p += hd.bytes[k];
    }
    const size_t nu = (size_t)(s.G.iny + 3) * (s.G.nz + 3);
    const double* u = (const double*)p;
    if (b->K->tbytes == 8) {
        TMX_CK(cudaMemcpyAsync(s.uin[0], u, nu * 8, cudaMemcpyHostToDevice, b->stream));
        TMX_CK(cudaMemcpyAsync(s.uin[1], u + nu, nu * 8, cudaMemcpyHostToDevice, b->stream));
    } else {
        std::vector<float> a(u, u + nu), c(u + nu, u + 2 * nu);
        TMX_CK(cudaMemcpyAsync(s.uin[0], a.data(), nu * 4, cudaMemcpyHostToDevice, b->stream));
        TMX_CK(cudaMemcpyAsync(s.uin[1], c.data(), nu * 4, cudaMemcpyHostToDevice, b->stream));
    }
    TMX_CK(cudaStreamSynchronize(b->stream));
    s.parity0 = b->parity;
    s.steps = hd.steps;
    return TMX_OK;
}

// Carve a slot for case c and either start it (buf == nullptr) or restore it.
int admit(tmx_batch* b, const tmx_case* c, const void* buf, long long size, int* slot)
{
    if (!b || !c || !slot) return fail(TMX_E_INVALID, "null argument");
    *slot = -1;
    int rc = check_case(*c);
    if (rc) return rc;
    if (c->precision != b->precision)
        return fail(TMX_E_INVALID, "case precision %d differs from the batch's %d", c->precision, b->precision);
    TMX_CK(cudaSetDevice(b->device));
    Slot s;
    s.c = *c;
    geometry_of(*c, s.G);
    physics_of(*c, s.P);
    const Carve cv = carve_of(s.G, b->precision);
    const long long off = b->arena.alloc(cv.total);
    if (off < 0)
        return fail(TMX_E_NOMEM, "batch budget: %lld bytes needed, %lld free (largest range %lld)", cv.total,
                    b->arena.free_bytes(), b->arena.largest());
    rc = boundary_list(s.G, s.nodes, s.cls, s.nface, nullptr, nullptr, &s.nzwall);
    if (rc) {
        b->arena.release(off, cv.total);
        return rc;
    }
    s.off = off;
    s.bytes = cv.total;
    char* p = b->arena_base + off;
    for (int q = 0; q < 2; q++) {
        s.pop[q] = p;
        p += cv.pop;
        s.rho[q] = p;
        p += cv.rho;
        s.uin[q] = p;
        p += cv.uin;
        if (cv.mom) {
            s.mom[q] = (float4*)p;
            p += cv.mom;
        }
    }
    s.mac = (double*)p;
    s.used = true;
    // the stream must be idle before a range of the arena is reused
    TMX_CK(cudaStreamSynchronize(b->stream));
    int m = -1;
    for (size_t i = 0; i < b->slots.size(); i++)
        if (!b->slots[i].used) {
            m = (int)i;
            break;
        }
    if (m < 0) {
        m = (int)b->slots.size();
        b->slots.emplace_back();
    }
    b->slots[m] = std::move(s);
    rc = buf ? restore_slot(b, b->slots[m], buf, size) : init_slot(b, b->slots[m]);
    if (rc) {
        b->arena.release(off, cv.total);
        b->slots[m] = Slot();
        return rc;
    }
    b->dirty = true;
    *slot = m;
    return TMX_OK;
}

}  // namespace

extern "C" {

int tmx_batch_add(tmx_batch* b, const tmx_case* c, int* slot) { return admit(b, c, nullptr, 0, slot); }

int tmx_batch_restore(tmx_batch* b, const tmx_case* c, const void* buf, long long bytes, int* slot)
{
    if (!buf) return fail(TMX_E_INVALID, "null checkpoint");
    return admit(b, c, buf, bytes, slot);
}

int tmx_batch_checkpoint(tmx_batch* b, int slot, void* buf, long long bytes)
{
    if (!b || !buf) return fail(TMX_E_INVALID, "null argument");
    if (!valid_slot(b, slot)) return fail(TMX_E_INVALID, "slot %d is not in the batch", slot);
    const Slot& s = b->slots[slot];
    long long sec[5];
    checkpoint_sections(s.G, b->precision, sec);
    if (bytes != checkpoint_total(sec))
        return fail(TMX_E_INVALID, "checkpoint buffer of %lld bytes, %lld needed", bytes, checkpoint_total(sec));
    TMX_CK(cudaSetDevice(b->device));
    TMX_CK(cudaStreamSynchronize(b->stream));
    CheckpointHeader hd{};
    std::memcpy(hd.magic, kCheckpointMagic, 8);
    hd.abi = TMX_ABI_VERSION;
    hd.precision = b->precision;
    hd.c = s.c;
    hd.steps = s.steps;
    hd.ps = s.G.ps;
    std::memcpy(hd.bytes, sec, sizeof sec);
    char* p = (char*)buf;
    std::memcpy(p, &hd, sizeof hd);
    p += sizeof hd;
    const int q = b->parity ^ s.parity0;  // the buffer set the next step reads
    const void* src[4] = {s.pop[q], s.rho[q], s.mom[q], s.mac};
    for (int k = 0; k < 4; k++) {
        if (sec[k]) TMX_CK(cudaMemcpy(p, src[k], (size_t)sec[k], cudaMemcpyDeviceToHost));
        p += sec[k];
    }
    std::vector<double> u1, u2;
    int rc = cached_inlet(s.c, b->stream, u1, u2);
    if (rc) return rc;
    std::memcpy(p, u1.data(), u1.size() * 8);
    std::memcpy(p + u1.size() * 8, u2.data(), u2.size() * 8);
    return TMX_OK;
}

int tmx_batch_checkpoint_size(const tmx_batch* b, int slot, long long* bytes)
{
    if (!b || !bytes) return fail(TMX_E_INVALID, "null argument");
    if (!valid_slot(b, slot)) return fail(TMX_E_INVALID, "slot %d is not in the batch", slot);
    long long sec[5];
    checkpoint_sections(b->slots[slot].G, b->precision, sec);
    *bytes = checkpoint_total(sec);
    return TMX_OK;
}

int tmx_batch_remove(tmx_batch* b, int slot)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    if (!valid_slot(b, slot)) return fail(TMX_E_INVALID, "slot %d is not in the batch", slot);
    TMX_CK(cudaSetDevice(b->device));
    TMX_CK(cudaStreamSynchronize(b->stream));
    Slot& s = b->slots[slot];
    b->arena.release(s.off, s.bytes);
    s = Slot();
    b->dirty = true;
    return TMX_OK;
}

int tmx_batch_step(tmx_batch* b, int nsteps, int write_macro_last)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    if (nsteps < 0) return fail(TMX_E_INVALID, "negative step count");
    TMX_CK(cudaSetDevice(b->device));
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    for (int s = 0; s < nsteps; s++) {
        int rc = step_one(b, (s == nsteps - 1 && write_macro_last) ? 1 : 0);
        if (rc) return rc;
    }
    for (auto& s : b->slots)
        if (s.used) s.steps += nsteps;
    return TMX_OK;
}

int tmx_batch_sync(tmx_batch* b)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    TMX_CK(cudaSetDevice(b->device));
    TMX_CK(cudaStreamSynchronize(b->stream));
    return TMX_OK;
}

int tmx_batch_slots(const tmx_batch* b, int* slots, int cap, int* n)
{
    if (!b || !n) return fail(TMX_E_INVALID, "null argument");
    int k = 0;
    for (size_t i = 0; i < b->slots.size(); i++)
        if (b->slots[i].used) {
            if (slots && k < cap) slots[k] = (int)i;
            k++;
        }
    *n = k;
    return TMX_OK;
}

long long tmx_batch_slot_steps(const tmx_batch* b, int slot)
{
    if (!b || !valid_slot(b, slot)) return -1;
    return b->slots[slot].steps;
}

int tmx_batch_outlet_im(tmx_batch* b, const int* slots, int n, double* im_out)
{
    if (!b || (n > 0 && (!slots || !im_out))) return fail(TMX_E_INVALID, "null argument");
    if (n <= 0) return TMX_OK;
    for (int e = 0; e < n; e++)
        if (!valid_slot(b, slots[e])) return fail(TMX_E_INVALID, "slot %d is not in the batch", slots[e]);
    TMX_CK(cudaSetDevice(b->device));
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    if (n > b->cap_im) {
        TMX_CK(cudaStreamSynchronize(b->stream));
        cudaFree(b->d_slots);
        cudaFree(b->d_im);
        b->d_slots = nullptr;
        b->d_im = nullptr;
        b->cap_im = 0;
        TMX_CK(cudaMalloc((void**)&b->d_slots, (size_t)n * sizeof(int)));
        TMX_CK(cudaMalloc((void**)&b->d_im, (size_t)n * 3 * sizeof(double)));
        b->cap_im = n;
    }
    TMX_CK(cudaMemcpyAsync(b->d_slots, slots, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    tmx::k_outlet_im_batch<<<n, 32, 0, b->stream>>>(b->d_desc, b->d_slots, n, b->d_im);
    TMX_CK(cudaGetLastError());
    TMX_CK(cudaMemcpyAsync(im_out, b->d_im, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    TMX_CK(cudaStreamSynchronize(b->stream));
    return TMX_OK;
}

int tmx_batch_health(tmx_batch* b, const int* slots, int n, int* bad)
{
    if (!b || (n > 0 && (!slots || !bad))) return fail(TMX_E_INVALID, "null argument");
    if (n <= 0) return TMX_OK;
    for (int e = 0; e < n; e++)
        if (!valid_slot(b, slots[e])) return fail(TMX_E_INVALID, "slot %d is not in the batch", slots[e]);
    TMX_CK(cudaSetDevice(b->device));
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    const int ns = (int)b->slots.size();
    if (ns > b->cap_flags) {
        TMX_CK(cudaStreamSynchronize(b->stream));
        cudaFree(b->d_flags);
        b->d_flags = nullptr;
        b->cap_flags = 0;
        TMX_CK(cudaMalloc((void**)&b->d_flags, (size_t)std::max(ns, 64) * sizeof(int)));
        b->cap_flags = std::max(ns, 64);
    }
    TMX_CK(cudaMemsetAsync(b->d_flags, 0, (size_t)ns * sizeof(int), b->stream));
    tmx::k_nonfinite_batch<<<b->sms * 4, 256, 0, b->stream>>>(b->d_desc, b->d_blocks, b->d_counts, b->d_flags);
    TMX_CK(cudaGetLastError());
    std::vector<int> flags((size_t)ns);
    TMX_CK(cudaMemcpyAsync(flags.data(), b->d_flags, flags.size() * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    TMX_CK(cudaStreamSynchronize(b->stream));
    for (int e = 0; e < n; e++) bad[e] = flags[(size_t)slots[e]];
    return TMX_OK;
}

int tmx_batch_fields(tmx_batch* b, int slot, int box, int field, double* host_out)
{
    if (!b || !host_out) return fail(TMX_E_INVALID, "null argument");
    if (!valid_slot(b, slot)) return fail(TMX_E_INVALID, "slot %d is not in the batch", slot);
    if (box < 0 || box > 1 || field < 0 || field > 6)
        return fail(TMX_E_INVALID, "box %d / field %d out of range", box, field);
    TMX_CK(cudaSetDevice(b->device));
    const Slot& s = b->slots[slot];
    const Geom& G = s.G;
    const int nx = G.nx[box], ny = G.ny[box], nz = G.nz;
    const size_t n = (size_t)nx * ny * nz;
    std::vector<double> stage(n);
    TMX_CK(cudaStreamSynchronize(b->stream));
    TMX_CK(cudaMemcpy(stage.data(), s.mac + (size_t)field * G.ps + G.base[box], n * sizeof(double),
                      cudaMemcpyDeviceToHost));
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) host_out[((size_t)i * ny + j) * nz + k] = stage[((size_t)k * ny + j) * nx + i];
    return TMX_OK;
}

int tmx_batch_info(const tmx_batch* b, long long out[8])
{
    if (!b || !out) return fail(TMX_E_INVALID, "null argument");
    long long nodes = 0;
    for (auto& s : b->slots)
        if (s.used) nodes += s.G.nnodes;
    out[0] = b->nactive;
    out[1] = nodes;
    out[2] = b->arena.capacity;
    out[3] = b->arena.free_bytes();
    out[4] = kBulkThreads[b->variant];
    out[5] = b->cells;
    out[6] = b->steps;
    out[7] = b->table_bytes;
    return TMX_OK;
}

int tmx_batch_set_shape(tmx_batch* b, int threads, int cells)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    int v = -1;
    for (int i = 0; i < 3; i++)
        if (kBulkThreads[i] == threads) v = i;
    if (v < 0) return fail(TMX_E_INVALID, "bulk threads per block must be 128, 256 or 512 (got %d)", threads);
    if (cells < threads || cells % threads) return fail(TMX_E_INVALID, "cells per block must be a multiple of %d", threads);
    TMX_CK(cudaSetDevice(b->device));
    TMX_CK(cudaStreamSynchronize(b->stream));
    if (v != b->variant || b->sweep) drop_graphs(b);
    b->variant = v;
    if (cells != b->cells || b->sweep) b->dirty = true;
    b->cells = cells;
    b->sweep = 0;
    return TMX_OK;
}

int tmx_batch_set_sweep(tmx_batch* b, int kind, int zchunk)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    if (!sweep_shape(kind)) return fail(TMX_E_INVALID, "tmx_batch_set_sweep: %d is not a sweep shape", kind);
    if (!b->K->moments) return fail(TMX_E_INVALID, "the sweep kernels are for the FP16 form only");
    if (zchunk < 1) return fail(TMX_E_INVALID, "planes per tile must be >= 1");
    TMX_CK(cudaSetDevice(b->device));
    TMX_CK(cudaStreamSynchronize(b->stream));
    if (kind != b->sweep) drop_graphs(b);
    if (kind != b->sweep || zchunk != b->zchunk) b->dirty = true;
    b->sweep = kind;
    b->zchunk = zchunk;
    return TMX_OK;
}

int tmx_batch_set_boundary(tmx_batch* b, int blocks_per_sm, int after)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    if (blocks_per_sm < 0) return fail(TMX_E_INVALID, "boundary blocks per SM must be >= 0 (got %d)", blocks_per_sm);
    if (after != 0 && after != 1) return fail(TMX_E_INVALID, "after must be 0 or 1 (got %d)", after);
    TMX_CK(cudaSetDevice(b->device));
    TMX_CK(cudaStreamSynchronize(b->stream));
    if (blocks_per_sm != b->bound_bps || after != b->bound_after) drop_graphs(b);
    b->bound_bps = blocks_per_sm;
    b->bound_after = after;
    set_grids(b);
    return TMX_OK;
}

int tmx_batch_boundary(const tmx_batch* b, int* blocks_per_sm, int* after)
{
    if (!b || !blocks_per_sm) return fail(TMX_E_INVALID, "null argument");
    *blocks_per_sm = b->grid_faces / std::max(1, b->sms);
    if (after) *after = (b->K->serial || b->bound_after) ? 1 : 0;
    return TMX_OK;
}

int tmx_batch_shape(const tmx_batch* b, int out[4])
{
    if (!b || !out) return fail(TMX_E_INVALID, "null argument");
    out[0] = b->sweep ? b->sweep : TMX_SHAPE_FLAT;
    out[1] = b->sweep ? sweep_shape(b->sweep)->threads() : kBulkThreads[b->variant];
    out[2] = b->cells;
    out[3] = b->zchunk;
    return TMX_OK;
}

// the sweep kernels' planes per tile tried by tmx_batch_tune
constexpr int kZChunkChoices[4] = {4, 8, 16, 32};

int tmx_batch_tune(tmx_batch* b, int steps_per_trial, int* threads_out, int* cells_out, double* ms_out)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    if (steps_per_trial <= 0) return fail(TMX_E_INVALID, "steps per trial must be positive");
    TMX_CK(cudaSetDevice(b->device));
    cudaEvent_t t0, t1;
    TMX_CK(cudaEventCreate(&t0));
    TMX_CK(cudaEventCreate(&t1));
    double best = 1e300;
    int bv = b->variant, bc = b->cells, bs = b->sweep, bz = b->zchunk;
    int rc = TMX_OK;
    // time steps_per_trial steps of the shape just set (after two steps that
    // capture its graphs and warm up)
    auto trial = [&](double& ms_step) {
        rc = tmx_batch_step(b, 2, 0);
        if (rc) return;
        cudaEventRecord(t0, b->stream);
        rc = tmx_batch_step(b, steps_per_trial, 0);
        cudaEventRecord(t1, b->stream);
        if (cudaEventSynchronize(t1) != cudaSuccess) rc = fail(TMX_E_CUDA, "tune: event wait failed");
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        ms_step = ms / steps_per_trial;
    };
    for (int v = 0; v < 3 && rc == TMX_OK; v++)
        for (int ci = 0; ci < 4 && rc == TMX_OK; ci++) {
            const int cells = kCellChoices[ci];
            if (cells < kBulkThreads[v]) continue;
            rc = tmx_batch_set_shape(b, kBulkThreads[v], cells);
            if (rc) break;
            double ms = 0;
            trial(ms);
            if (rc == TMX_OK && ms < best) {
                best = ms;
                bv = v;
                bc = cells;
                bs = 0;
            }
        }
    if (b->K->moments)
        for (int kind = TMX_SHAPE_SWEEP8; kind <= TMX_SHAPE_SWEEP4; kind++)
            for (int zi = 0; zi < 4 && rc == TMX_OK; zi++) {
                rc = tmx_batch_set_sweep(b, kind, kZChunkChoices[zi]);
                if (rc) break;
                double ms = 0;
                trial(ms);
                if (rc == TMX_OK && ms < best) {
                    best = ms;
                    bs = kind;
                    bz = kZChunkChoices[zi];
                }
            }
    // the boundary kernels with the chosen interior kernel (they share the
    // SMs with it): a persistent grid of 1, 2, 4 blocks per SM or as many as
    // fit, beside the interior kernel or (reduced-precision forms) before it
    int bb = b->bound_bps, ba = b->bound_after;
    if (rc == TMX_OK) rc = tmx_batch_set_shape(b, kBulkThreads[bv], bc);
    if (rc == TMX_OK && bs) rc = tmx_batch_set_sweep(b, bs, bz);
    const int bchoices[4] = {1, 2, 4, 0};
    for (int after = 0; after < (b->K->serial ? 1 : 2) && rc == TMX_OK; after++)
        for (int i = 0; i < 4 && rc == TMX_OK; i++) {
            if (bchoices[i] >= b->bound_fit) continue;  // the same grid as 0
            rc = tmx_batch_set_boundary(b, bchoices[i], after);
            if (rc) break;
            double ms = 0;
            trial(ms);
            if (rc == TMX_OK && ms < best) {
                best = ms;
                bb = bchoices[i];
                ba = after;
            }
        }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    rc = tmx_batch_set_boundary(b, bb, ba);
    if (rc) return rc;
    // the trials advanced the mixers: start every one of them again
    TMX_CK(cudaStreamSynchronize(b->stream));
    for (auto& s : b->slots)
        if (s.used) {
            rc = init_slot(b, s);
            if (rc) return rc;
        }
    b->dirty = true;
    TMX_CK(cudaStreamSynchronize(b->stream));
    if (threads_out) *threads_out = bs ? sweep_shape(bs)->threads() : kBulkThreads[bv];
    if (cells_out) *cells_out = bs ? sweep_shape(bs)->threads() * bz : bc;
    if (ms_out) *ms_out = best;
    return TMX_OK;
}

int tmx_batch_step_timed(tmx_batch* b, int nsteps, double* ms_interior, double* ms_boundary, double* ms_total)
{
    if (!b) return fail(TMX_E_INVALID, "null batch");
    if (nsteps <= 0) return fail(TMX_E_INVALID, "nsteps must be positive");
    TMX_CK(cudaSetDevice(b->device));
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    std::vector<cudaEvent_t> ev((size_t)nsteps * 4, nullptr);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaError_t e = cudaSuccess;
    for (auto& x : ev)
        if (e == cudaSuccess) e = cudaEventCreate(&x);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    int rc = e == cudaSuccess ? TMX_OK : fail(TMX_E_CUDA, "tmx_batch_step_timed: %s", cudaGetErrorString(e));
    if (rc == TMX_OK && cudaEventRecord(t0, b->stream) != cudaSuccess) rc = fail(TMX_E_CUDA, "event record failed");
    int done = 0;
    for (; done < nsteps && rc == TMX_OK; done++) {
        rc = enqueue(b, b->parity, 0, &ev[(size_t)done * 4]);
        if (rc == TMX_OK) {
            b->parity ^= 1;
            b->steps++;
        }
    }
    for (auto& s : b->slots)
        if (s.used) s.steps += done - (rc == TMX_OK ? 0 : 1);
    double si = 0, sb = 0;
    float tot = 0;
    if (rc == TMX_OK) {
        cudaEventRecord(t1, b->stream);
        if (cudaEventSynchronize(t1) != cudaSuccess) rc = fail(TMX_E_CUDA, "tmx_batch_step_timed: event wait failed");
    }
    for (int s = 0; s < nsteps && rc == TMX_OK; s++) {
        float a = 0, c = 0;
        cudaEventElapsedTime(&a, ev[(size_t)s * 4], ev[(size_t)s * 4 + 1]);
        cudaEventElapsedTime(&c, ev[(size_t)s * 4 + 2], ev[(size_t)s * 4 + 3]);
        si += a;
        sb += c;
    }
    if (rc == TMX_OK) cudaEventElapsedTime(&tot, t0, t1);
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (rc) return rc;
    if (ms_interior) *ms_interior = si;
    if (ms_boundary) *ms_boundary = sb;
    if (ms_total) *ms_total = tot;
    return TMX_OK;
}

int tmx_batch_time_steps(tmx_batch* b, int nsteps, double* ms)
{
    if (!b || !ms) return fail(TMX_E_INVALID, "null argument");
    if (nsteps <= 0) return fail(TMX_E_INVALID, "nsteps must be positive");
    TMX_CK(cudaSetDevice(b->device));
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    cudaEvent_t t0, t1;
    TMX_CK(cudaEventCreate(&t0));
    TMX_CK(cudaEventCreate(&t1));
    TMX_CK(cudaEventRecord(t0, b->stream));
    int rc = tmx_batch_step(b, nsteps, 0);
    TMX_CK(cudaEventRecord(t1, b->stream));
    TMX_CK(cudaEventSynchronize(t1));
    float f = 0;
    cudaEventElapsedTime(&f, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    *ms = f;
    return rc;
}

void tmx_batch_destroy(tmx_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    cudaFree(b->d_desc);
    cudaFree(b->d_blocks);
    cudaFree(b->d_faces);
    cudaFree(b->d_edges);
    cudaFree(b->d_tiles);
    cudaFree(b->d_counts);
    cudaFree(b->d_slots);
    cudaFree(b->d_im);
    cudaFree(b->d_flags);
    cudaFree(b->arena_base);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->join2) cudaEventDestroy(b->join2);
    if (b->aux) cudaStreamDestroy(b->aux);
    if (b->aux2) cudaStreamDestroy(b->aux2);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // extern "C"
