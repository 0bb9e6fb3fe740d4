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
    void (*faces)(tmx::StepPtrs, const int*, const unsigned char*, int, Geom, Phys, int);
    void (*edges)(tmx::StepPtrs, const int*, const unsigned char*, int, Geom, Phys, int);
    int sbytes, tbytes;
    bool moments;  // the form stores per-node FP32 moments next to the populations
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
// first nface entries are face classes.  Returns TMX_OK or a failure code.
int boundary_list(const Geom& G, std::vector<int>& nodes, std::vector<unsigned char>& cls, int& nface,
                  std::vector<int>* class_count);
// Inlet profiles Uin1, Uin2 ((iny+3) x (nz+3)) as the reference computes them:
// the duct series (which depends on iny and nz only) and its mean, then the
// scaling to umean and the shifts.
void inlet_profile(const tmx_case& c, std::vector<double>& U1, std::vector<double>& U2);
void inlet_series(int iny, int nz, std::vector<double>& raw, double& average);
void inlet_scale(const tmx_case& c, const std::vector<double>& raw, double average, std::vector<double>& U1,
                 std::vector<double>& U2);

}  // namespace tmx_host
