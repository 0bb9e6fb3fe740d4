// tmx_kernels.cuh -- launch declarations of the kernels in tmx_kernels.cu.
#pragma once
#include "tmx_device.cuh"

namespace tmx {

__global__ void k_init(double* __restrict__ Pout, double* __restrict__ R, double* __restrict__ Mac, Geom G, Phys P,
                       double rho0);
__global__ void k_bulk(const double* __restrict__ Pin, double* __restrict__ Pout, double* __restrict__ Rcur,
                       double* __restrict__ Mac, Geom G, Phys P, int write_macro);
constexpr int kBoundaryThreadsHost = 128;  // block size of k_boundary
// inlet/outlet/wall-face nodes and edge/corner nodes of the boundary list
__global__ void k_boundary_faces(const double* __restrict__ Pin, double* __restrict__ Pout,
                                 const double* __restrict__ Rprev, double* __restrict__ Rcur, double* __restrict__ Mac,
                                 const int* __restrict__ bnode, const unsigned char* __restrict__ bcls, int nb,
                                 const double* __restrict__ uin1, const double* __restrict__ uin2, Geom G, Phys P,
                                 int write_macro);
__global__ void k_boundary_edges(const double* __restrict__ Pin, double* __restrict__ Pout,
                                 const double* __restrict__ Rprev, double* __restrict__ Rcur, double* __restrict__ Mac,
                                 const int* __restrict__ bnode, const unsigned char* __restrict__ bcls, int nb,
                                 const double* __restrict__ uin1, const double* __restrict__ uin2, Geom G, Phys P,
                                 int write_macro);
__global__ void k_mixing_rows(const double* __restrict__ Mac, Geom G, double* __restrict__ stats);
__global__ void k_sums(const double* __restrict__ Mac, Geom G, double* __restrict__ partial);

}  // namespace tmx
