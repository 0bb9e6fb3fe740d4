// tmx_kernels.cuh -- launch declarations of the kernels in tmx_kernels.cu
// (FP64 form, reductions) and tmx_kernels_lp.cu (FP32 / FP16-storage forms).
// Population, density and inlet-profile buffers are typed by the form
// (double / float / __half storage; double / float arithmetic), hence void*.
#pragma once
#include "tmx_device.cuh"

namespace tmx {

// Buffers of one step (populations in/out, boundary densities previous/this
// step, macroscopic fields, FP16-form moments previous/this step, inlet
// profiles); the kernels cast to the form's types.
struct StepPtrs {
    const void* pin;
    void* pout;
    const void* rprev;
    void* rcur;
    double* mac;
    const float4* mprev;
    float4* mcur;
    const void* uin1;
    const void* uin2;
};

constexpr int kBoundaryThreadsHost = 128;  // block size of the boundary kernels
constexpr int kBoundaryLanesHost = 4;      // threads per boundary node (one per field)
// A batched boundary block takes kListAlign consecutive list entries at a
// time; the batch pads each mixer's part of a list to a multiple of it.
constexpr int kListAlign = kBoundaryThreadsHost / kBoundaryLanesHost;

#define TMX_DECLARE_STEP_KERNELS(NAME)                                                                          \
    __global__ void k_init_##NAME(StepPtrs X, Geom G, Phys P, double rho0);                                     \
    __global__ void k_bulk_##NAME(StepPtrs X, Geom G, Phys P, int write_macro);
#define TMX_DECLARE_BOUNDARY_KERNELS(NAME)                                                                      \
    __global__ void k_bfaces_##NAME(StepPtrs X, const int* bnode, const unsigned char* bcls, int nb, Geom G,    \
                                    Phys P, int write_macro);                                                   \
    __global__ void k_bedges_##NAME(StepPtrs X, const int* bnode, const unsigned char* bcls, int nb, Geom G,    \
                                    Phys P, int write_macro);

TMX_DECLARE_STEP_KERNELS(f64)
TMX_DECLARE_STEP_KERNELS(f32)
TMX_DECLARE_STEP_KERNELS(f16)
TMX_DECLARE_BOUNDARY_KERNELS(f32)
TMX_DECLARE_BOUNDARY_KERNELS(f16)
__global__ void k_bound_f64(StepPtrs X, const int* bnode, const unsigned char* bcls, int nf, int ne, int eblocks,
                            Geom G, Phys P, int write_macro);
__global__ void k_walls_f64(StepPtrs X, const int* wnode, const unsigned char* wcls, int nw, Geom G, Phys P,
                            int write_macro);

// One mixer of a batch: its buffers for either parity of the batch's step
// counter, its geometry and its physics constants (device memory, read by
// the batched kernels).
struct MixerDesc {
    StepPtrs X[2];
    Geom G;
    Phys P;
};

// Batched step kernels: one launch covers every mixer of a batch.
//   bulk    a persistent grid walks a list of cell blocks {mixer, first
//           node, node count, 0}; NT threads per block (128, 256 or 512).
//   faces / edges   boundary-node lists of {node, mixer * 256 + class},
//           four threads per node, persistent grid; each mixer's part
//           starts at a multiple of kListAlign, padded with node -1.
// counts[0..2] = number of cell blocks, face nodes, edge nodes (device
// memory, so that captured graphs stay valid when the batch changes).
#define TMX_DECLARE_BATCH_KERNELS(NAME)                                                                           \
    __global__ void k_bulk_batch128_##NAME(const MixerDesc* D, const int4* blocks, const int* counts, int parity, \
                                           int write_macro);                                                      \
    __global__ void k_bulk_batch256_##NAME(const MixerDesc* D, const int4* blocks, const int* counts, int parity, \
                                           int write_macro);                                                      \
    __global__ void k_bulk_batch512_##NAME(const MixerDesc* D, const int4* blocks, const int* counts, int parity, \
                                           int write_macro);                                                      \
    __global__ void k_bfaces_batch_##NAME(const MixerDesc* D, const int2* list, const int* counts, int parity,    \
                                          int write_macro);                                                       \
    __global__ void k_bedges_batch_##NAME(const MixerDesc* D, const int2* list, const int* counts, int parity,    \
                                          int write_macro);

TMX_DECLARE_BATCH_KERNELS(f64)
TMX_DECLARE_BATCH_KERNELS(f32)
TMX_DECLARE_BATCH_KERNELS(f16)

// The FP16 form's interior by tiles of 32 x TY nodes swept through z
// (tmx_engine.cuh sweep_tile): tiles[t] = {mixer * 2 + box, x0 | y0 << 16,
// z0 | z1 << 16}; the single-mixer kernels take mixer 0, the batched ones read
// the tile count from counts[3].  Dynamic shared memory: sweep_smem_host(TY).
#define TMX_DECLARE_SWEEP(SUFFIX)                                                                               \
    __global__ void k_sweep##SUFFIX##_f16(StepPtrs X, Geom G, Phys P, int write_macro, const int4* tiles,     \
                                          int ntiles);                                                        \
    __global__ void k_sweep_batch##SUFFIX##_f16(const MixerDesc* D, const int4* tiles, const int* counts,     \
                                                int parity, int write_macro);
TMX_DECLARE_SWEEP(8)
TMX_DECLARE_SWEEP(4)
constexpr int sweep_smem_host(int ty) { return 2 * 4 * (ty + 2) * 34 * 16; }

// Outlet mixing quality of batch mixers: for entry e, mixer slots[e], the
// I_A, I_B, I_C of mixing row 1 (the first row of tmx_mixing) into
// out[3e..3e+2], with the arithmetic of k_mixing_rows and its finish.
__global__ void k_outlet_im_batch(const MixerDesc* D, const int* slots, int n, double* out);

// Health of batch mixers: flags[m] |= 1 for every mixer m with a non-finite
// macroscopic value (density, velocity or concentration) in the last fields
// written, over the batch's cell-block list (counts[0] blocks).
__global__ void k_nonfinite_batch(const MixerDesc* D, const int4* blocks, const int* counts, int* flags);

__global__ void k_mixing_rows(const double* __restrict__ Mac, Geom G, double* __restrict__ stats);
__global__ void k_sums(const double* __restrict__ Mac, Geom G, double* __restrict__ partial);
// The inlet duct series of the reduced-precision forms, computed on the device.
__global__ void k_inlet_series(int iny, int nz, double* __restrict__ raw);
// Pressure and specific power of one mixer (layout of out: tmx_kernels.cu).
__global__ void k_pressure_power(const double* __restrict__ Mac, Geom G, double tau, double* __restrict__ out);

// Fixed scratch of tmx_mixing_static: kMixStaticRows rows of 9 statistics
// followed by kMixStaticRows finished rows of 7 numbers (512 KiB per device).
constexpr int kMixStaticRows = 4096;
__global__ void k_mixing_finish(const double* __restrict__ stats, Geom G, double* __restrict__ rows);
// Device address of that scratch on the current device.
cudaError_t mixing_static_scratch(double** ptr);

}  // namespace tmx
