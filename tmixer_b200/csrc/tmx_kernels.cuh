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

#define TMX_DECLARE_STEP_KERNELS(NAME)                                                                          \
    __global__ void k_init_##NAME(StepPtrs X, Geom G, Phys P, double rho0);                                     \
    __global__ void k_bulk_##NAME(StepPtrs X, Geom G, Phys P, int write_macro);                                 \
    __global__ void k_bfaces_##NAME(StepPtrs X, const int* bnode, const unsigned char* bcls, int nb, Geom G,    \
                                    Phys P, int write_macro);                                                   \
    __global__ void k_bedges_##NAME(StepPtrs X, const int* bnode, const unsigned char* bcls, int nb, Geom G,    \
                                    Phys P, int write_macro);

TMX_DECLARE_STEP_KERNELS(f64)
TMX_DECLARE_STEP_KERNELS(f32)
TMX_DECLARE_STEP_KERNELS(f16)

__global__ void k_mixing_rows(const double* __restrict__ Mac, Geom G, double* __restrict__ stats);
__global__ void k_sums(const double* __restrict__ Mac, Geom G, double* __restrict__ partial);

// Fixed scratch of tmx_mixing_static: kMixStaticRows rows of 9 statistics
// followed by kMixStaticRows finished rows of 7 numbers (512 KiB per device).
constexpr int kMixStaticRows = 4096;
__global__ void k_mixing_finish(const double* __restrict__ stats, Geom G, double* __restrict__ rows);
// Device address of that scratch on the current device.
cudaError_t mixing_static_scratch(double** ptr);

}  // namespace tmx
