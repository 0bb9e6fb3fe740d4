// tmx_kernels.cuh -- launch declarations of the kernels in tmx_kernels.cu
// (FP64 form, reductions) and tmx_kernels_lp.cu (FP32 / FP16-storage forms).
// Population, density and inlet-profile buffers are typed by the form
// (double / float / __half storage; double / float arithmetic), hence void*.
#pragma once
#include "tmx_device.cuh"

namespace tmx {

constexpr int kBoundaryThreadsHost = 128;  // block size of the boundary kernels

#define TMX_DECLARE_STEP_KERNELS(NAME)                                                                          \
    __global__ void k_init_##NAME(void* Pout, void* R, double* Mac, Geom G, Phys P, double rho0);              \
    __global__ void k_bulk_##NAME(const void* Pin, void* Pout, void* Rcur, double* Mac, Geom G, Phys P,         \
                                  int write_macro);                                                             \
    __global__ void k_bfaces_##NAME(const void* Pin, void* Pout, const void* Rprev, void* Rcur, double* Mac,    \
                                    const int* bnode, const unsigned char* bcls, int nb, const void* uin1,      \
                                    const void* uin2, Geom G, Phys P, int write_macro);                         \
    __global__ void k_bedges_##NAME(const void* Pin, void* Pout, const void* Rprev, void* Rcur, double* Mac,    \
                                    const int* bnode, const unsigned char* bcls, int nb, const void* uin1,      \
                                    const void* uin2, Geom G, Phys P, int write_macro);

TMX_DECLARE_STEP_KERNELS(f64)
TMX_DECLARE_STEP_KERNELS(f32)
TMX_DECLARE_STEP_KERNELS(f16)

__global__ void k_mixing_rows(const double* __restrict__ Mac, Geom G, double* __restrict__ stats);
__global__ void k_sums(const double* __restrict__ Mac, Geom G, double* __restrict__ partial);

}  // namespace tmx
