// Batched truncated free-tensor product: the building block of ft_fma,
// ft_mul, in-place multiply and the Horner series (exp, fmexp, log).
#pragma once

#include "common.cuh"

namespace rpyb {

// One launch computes, for every row b and every output level
// k in [klo, khi] (k >= 1),
//
//   out_k = base_k + scale_k * sum_{p = pmax_k .. pmin_k} L_p (x) R_{k-p}
//
// where base_k is the old out_k (accumulate) or addend_k (or 0), L_0 may be
// overridden by a constant, and level 0 is handled by a small rule set.
struct ProductSpec {
    int klo = 1, khi = 0;            // output levels (>= 1); empty if khi < klo
    int pmin[kMaxDepth + 1] = {};    // per output level: lhs degree range
    int pmax[kMaxDepth + 1] = {};
    double scale[kMaxDepth + 1] = {};  // per-level multiplier of the sum
    bool accumulate = false;         // base = old out (scale must be 1)
    bool lhs0_from_mem = true;       // L_0 = (lhs[0] if from_mem else 0) + lhs0_add
    double lhs0_add = 0.0;
    // level-0 rule: out[0] = base0 + l0_const + (l0_prod ? scale0 * L0 * R0 : 0)
    // base0: 0 -> 0, 1 -> old out[0], 2 -> addend[0]; l0_write false = untouched
    bool l0_write = false;
    int l0_base = 0;
    double l0_const = 0.0;
    bool l0_prod = false;
    double scale0 = 1.0;
};

struct ProductRows {
    void* out = nullptr;
    const void* lhs = nullptr;
    const void* rhs = nullptr;
    const void* addend = nullptr;   // nullable (assign mode)
    int64_t ld_out = 0, ld_lhs = 0, ld_rhs = 0, ld_add = 0;
    const int64_t* out_idx = nullptr;  // nullable row gathers
    const int64_t* lhs_idx = nullptr;
    const int64_t* rhs_idx = nullptr;
    int64_t batch = 0;
};

// dtype RPYB_F64 (double), RPYB_F32 (float, compensated accumulation) or
// kMixedF64F32 (double output and left factor, float right factor).
constexpr int kMixedF64F32 = 2;
int launch_product(int dtype, const Geometry& g, const ProductSpec& spec,
                   const ProductRows& rows, cudaStream_t stream);

// Elementwise helpers used by the Horner drivers.
int launch_convert_rows(int dst_dtype, void* dst, int64_t ld_dst, int src_dtype,
                        const void* src, int64_t ld_src, int64_t cols, int64_t batch,
                        cudaStream_t stream);

}  // namespace rpyb
