// Shared definitions for the B200 tensor-algebra kernels and their host
// launchers: error plumbing, basis geometry and compensated arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/rpyb.h"

namespace rpyb {

constexpr int kMaxDepth = 16;

// ---------------------------------------------------------------- errors --
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t err, const char* what);

#define RPYB_CUDA(call)                                                   \
    do {                                                                  \
        cudaError_t rpyb_err_ = (call);                                   \
        if (rpyb_err_ != cudaSuccess) return ::rpyb::cuda_fail(rpyb_err_, #call); \
    } while (0)

// ---------------------------------------------------------------- basis --
// Degree-major layout of a dense free tensor: level k starts at
// degree_begin[k] = (d^k - 1)/(d - 1) and holds d^k words
// (roughpy/compute/_src/call_config.cpp:117-119 builds the same table).
struct Geometry {
    int32_t width = 0;
    int32_t depth = 0;
    int64_t db[kMaxDepth + 2] = {};   // degree_begin
    int64_t pw[kMaxDepth + 1] = {};   // width^k
    int64_t size() const { return db[depth + 1]; }
};

// Fills g; returns 0 or sets the error and returns RPYB_E_INVALID.
int make_geometry(int32_t width, int32_t depth, Geometry& g);

// Clamp a roughpy-style max degree (-1 or > depth means depth).
inline int32_t clamp_max_degree(int32_t d, int32_t depth)
{
    return (d < 0 || d > depth) ? depth : d;
}

// Stream-ordered scratch: uses the caller's workspace when given, otherwise
// takes memory from the library's per-device pool (cudaMallocFromPoolAsync)
// and releases it with cudaFreeAsync; the pool keeps freed memory for reuse.
class Scratch {
public:
    Scratch(void* ws, size_t ws_bytes, cudaStream_t s) : ws_(ws), cap_(ws_bytes), s_(s) {}
    ~Scratch();
    // Returns 0 and sets *p, or an error code.
    int get(size_t bytes, void** p);

private:
    void* ws_;
    size_t cap_;
    cudaStream_t s_;
    void* owned_ = nullptr;
};

// ----------------------------------------------- compensated arithmetic --
// Error-free transformations (Knuth two-sum, FMA two-product).  The
// explicit _rn intrinsics stop the compiler from contracting a product into
// a later addition, which would break the exactness the transformations
// rely on.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = __fadd_rn(a, b);
    float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e)
{
    p = __fmul_rn(a, b);
    e = __fmaf_rn(a, b, -p);
}

// Double-float accumulator: value = hi + lo.
struct DF {
    float hi, lo;
};

__device__ __forceinline__ void df_add_prod(DF& acc, float a, float b)
{
    float p, pe, s, se;
    two_prod(a, b, p, pe);
    two_sum(acc.hi, p, s, se);
    acc.hi = s;
    acc.lo = __fadd_rn(acc.lo, __fadd_rn(se, pe));
}

__device__ __forceinline__ float df_value(const DF& a) { return __fadd_rn(a.hi, a.lo); }

// Most pieces the dissection of one interval can produce.
constexpr int kMaxDyadicPieces = 2 * (4 * 64 + 1);

// Dissects the clopen interval [inf, sup) at resolution tol into maximal
// dyadic pieces k / 2^p, in order; writes at most kMaxDyadicPieces and returns
// their number, or a negative error code for an invalid interval or resolution.
int dissect_clopen(double inf, double sup, int32_t tol, int64_t* k, int32_t* p);

}  // namespace rpyb
