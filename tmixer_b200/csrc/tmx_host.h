// tmx_host.h -- host-side pieces shared by the single-mixer handle
// (tmx_api.cu) and the batched engine (tmx_batch.cu): error reporting, the
// kernel table of each precision form, and the translation of a tmx_case
// into device geometry, physics constants, boundary lists and inlet
// profiles.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/tmx.h"
#include "tmx_kernels.cuh"

namespace tmx_host {

using tmx::Geom;
using tmx::Phys;

// Record the error text of the calling thread (returned by tmx_last_error)
// and return code.
int fail(int code, const char* fmt, ...);
const char* last_error();

#define TMX_CK(call)                                                                                    \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return ::tmx_host::fail(TMX_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                                    __LINE__);                                                          \
    } while (0)

// the step kernels of one form
struct StepKernels {
    void (*init)(tmx::StepPtrs, Geom, Phys, double);
    void (*bulk)(tmx::StepPtrs, Geom, Phys, int);
    // the face and edge lists as two launches (forms whose bulk runs beside them)
    void (*faces)(tmx::StepPtrs, const int*, const unsigned char*, int, Geom, Phys, int);
    void (*edges)(tmx::StepPtrs, const int*, const unsigned char*, int, Geom, Phys, int);
    // faces and edges in one launch (serial forms only)
    void (*bound)(tmx::StepPtrs, const int*, const unsigned char*, int, int, int, Geom, Phys, int);
    // the wall faces, one thread per node (null: the face kernel takes them)
    void (*walls)(tmx::StepPtrs, const int*, const unsigned char*, int, Geom, Phys, int);
    int sbytes, tbytes;
    bool moments;  // the form stores per-node FP32 moments next to the populations
    bool serial;   // the bulk kernel runs after the boundary kernels, not beside them
};
extern const StepKernels kForms[3];

constexpr int kSumBlocks = 592;

// Validation of a case (the body of tmx_case_check).
int check_case(const tmx_case& c);
void geometry_of(const tmx_case& c, Geom& G);
void physics_of(const tmx_case& c, Phys& P);
// Device bytes of one single-mixer handle.
long long footprint(const Geom& G, long long nb, int precision);
long long boundary_count(const Geom& G);
// Class of a boundary node (tmx_classes.h), -1 for a node no case covers.
int classify(const Geom& G, int b, int i, int j, int k);
// Boundary nodes sorted faces first, then by class, then by node index; the
// first nface entries are face classes.  With nwall the wall faces
// (tmx::wall_class) come last, in node order, and *nwall counts them.
// Without nwall and with nzwall (the FP32 and FP16 forms), the z wall faces
// (K_FACE_Z1, K_FACE_ZT) come last among the faces and *nzwall counts them:
// each lies above or below an interior node and each interior node of planes
// 2 and nz - 1 has one (checked; an internal error otherwise), and the sweep
// kernels update them (zwall_node).  Without interior nodes (nz < 3) they
// stay in place and *nzwall is 0.  Returns TMX_OK or a failure code.
int boundary_list(const Geom& G, std::vector<int>& nodes, std::vector<unsigned char>& cls, int& nface,
                  std::vector<int>* class_count, int* nwall, int* nzwall);
// Inlet profiles Uin1, Uin2 ((iny+3) x (nz+3)) as the reference computes them:
// the duct series (which depends on iny and nz only) and its mean, then the
// scaling to umean and the shifts.
void inlet_profile(const tmx_case& c, std::vector<double>& U1, std::vector<double>& U2);
void inlet_series(int iny, int nz, std::vector<double>& raw, double& average);
// The same series computed on the current device (k_inlet_series) with the
// host's summation of the mean; for the reduced-precision forms.
int inlet_series_device(int iny, int nz, cudaStream_t stream, std::vector<double>& raw, double& average);
// The inlet profiles of a case in its form: the host series for FP64 (the
// reference's bits), the device series otherwise.
int inlet_profile_form(const tmx_case& c, cudaStream_t stream, std::vector<double>& U1, std::vector<double>& U2);
void inlet_scale(const tmx_case& c, const std::vector<double>& raw, double average, std::vector<double>& U1,
                 std::vector<double>& U2);

// The FP16 form's sweep kernels by shape (include/tmx.h TMX_SHAPE_SWEEP*):
// tile height, the single-mixer and batched kernels and their dynamic shared
// memory.
struct SweepShape {
    int kind, ty;
    void (*single)(tmx::StepPtrs, Geom, Phys, int, const int4*, int);
    void (*batch)(const tmx::MixerDesc*, const int4*, const int*, int, int);
    int threads() const { return 32 * ty; }
    int smem() const { return tmx::sweep_smem_host(ty); }
};
inline const SweepShape* sweep_shape(int kind)
{
    static const SweepShape shapes[] = {
        {TMX_SHAPE_SWEEP8, 8, tmx::k_sweep8_f16, tmx::k_sweep_batch8_f16},
        {TMX_SHAPE_SWEEP4, 4, tmx::k_sweep4_f16, tmx::k_sweep_batch4_f16},
    };
    for (const SweepShape& e : shapes)
        if (e.kind == kind) return &e;
    return nullptr;
}
// Allow each sweep kernel its dynamic shared memory on the current device
// (idempotent); returns the first error.
inline cudaError_t sweep_allow_smem()
{
    for (int kind = TMX_SHAPE_SWEEP8; kind <= TMX_SHAPE_SWEEP4; kind++) {
        const SweepShape* sh = sweep_shape(kind);
        cudaError_t e = cudaFuncSetAttribute((const void*)sh->single, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             sh->smem());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute((const void*)sh->batch, cudaFuncAttributeMaxDynamicSharedMemorySize, sh->smem());
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Tiles of the sweep kernels (tmx_engine.cuh sweep_tile) for one mixer:
// {mixer * 2 + box, x0 | y0 << 16, z0 | z1 << 16, 0}, 32 x ty nodes of a box
// (0-based x0, y0) over the interior planes z0 .. z1-1 (zchunk at most),
// z-chunks outermost.
inline void sweep_tiles(const Geom& G, int mixer, int ty, int zchunk, std::vector<int4>& out)
{
    for (int z0 = 2; z0 <= G.nz - 1; z0 += zchunk) {
        const int z1 = z0 + zchunk < G.nz ? z0 + zchunk : G.nz;
        for (int b = 0; b < 2; b++)
            for (int y0 = 0; y0 < G.ny[b]; y0 += ty)
                for (int x0 = 0; x0 < G.nx[b]; x0 += 32)
                    out.push_back(make_int4(mixer * 2 + b, x0 | (y0 << 16), z0 | (z1 << 16), 0));
    }
}

// Checkpoint layout (tmx_checkpoint, tmx_batch_checkpoint): this header, then
// the sections in the order of `bytes`: the population buffer the next step
// reads (76 planes of ps values of the storage type), the previous step's
// densities (4 planes, arithmetic type), the FP16 form's moment records
// (2 float4 per node, or nothing), the macroscopic fields (7 FP64 planes) and
// the two inlet profiles ((iny+3)(nz+3) FP64 values each).
// "TMXCKPT2": FP16 records {(rho, cA, cB, cC), (ux, uy, uz, omt)};
// "TMXCKPT1" (refused) had {(rho, ux, uy, uz), (cA, cB, cC, omt)}
constexpr char kCheckpointMagic[9] = "TMXCKPT2";
struct CheckpointHeader {
    char magic[8];  // kCheckpointMagic
    int abi;
    int precision;
    tmx_case c;
    long long steps;
    long long ps;
    long long bytes[5];
};
inline void checkpoint_sections(const Geom& G, int precision, long long bytes[5])
{
    const StepKernels& K = kForms[precision];
    bytes[0] = 76LL * G.ps * K.sbytes;
    bytes[1] = 4LL * G.ps * K.tbytes;
    bytes[2] = K.moments ? 2LL * G.ps * 16 : 0;
    bytes[3] = 7LL * G.ps * 8;
    bytes[4] = 2LL * (G.iny + 3) * (G.nz + 3) * 8;
}
inline long long checkpoint_total(const long long bytes[5])
{
    return (long long)sizeof(CheckpointHeader) + bytes[0] + bytes[1] + bytes[2] + bytes[3] + bytes[4];
}
// Check a checkpoint against a case; TMX_OK or TMX_E_INVALID with a message.
int checkpoint_check(const void* buf, long long size, const tmx_case& c, const Geom& G);

}  // namespace tmx_host
