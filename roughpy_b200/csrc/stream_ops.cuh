// Building blocks shared by the stream runtimes (dyadic tree, piecewise
// abelian streams) and the signature derivative: Lie maps cached on the
// device, ordered row products, and the log-signature / signature finish of
// a batch of group-like products.
#pragma once

#include <vector>

#include "common.cuh"

namespace rpyb {

// CSR form of both Lie maps on the current device, uploaded once per
// (device, width, depth) and kept for the life of the process.
struct LieMapsDev {
    int device = -1;
    int32_t width = 0, depth = 0;
    int64_t lie_dim = 0;
    const int64_t* l2t_ptr = nullptr;   // tensor_size rows x lie_dim
    const int64_t* l2t_idx = nullptr;
    const double* l2t_val = nullptr;
    const int64_t* t2l_ptr = nullptr;   // lie_dim rows x tensor_size
    const int64_t* t2l_idx = nullptr;
    const double* t2l_val = nullptr;
    // t2l packed for the shared-memory projection kernel (null when a column
    // does not fit 16 bits or the number of distinct values 13 bits).  Rows sorted by
    // entry count, in groups of 32 (one per warp lane), each group padded to
    // its longest row; entry j of lane l of group g is t2l_ent[t2l_goff[g] +
    // 32 j + l] = 8 * column | (value id << 19), the distinct values (and a zero
    // for the padding) in t2l_tab; t2l_perm[32 g + l] is the lane's row, or
    // 0xffffffff past the last row.
    const uint32_t* t2l_goff = nullptr;   // groups + 1
    const uint32_t* t2l_ent = nullptr;
    const uint32_t* t2l_perm = nullptr;   // 32 * groups
    const double* t2l_tab = nullptr;
    int64_t t2l_slots = 0, t2l_groups = 0, t2l_ntab = 0;
};
int lie_maps_device(const Geometry& g, const LieMapsDev** out);

// lie[b] <- t2l(x[b]) for m rows (assigning; dtype RPYB_F32 or RPYB_F64 for
// both, float64 arithmetic)
int lie_project(int dtype, const Geometry& g, const LieMapsDev& maps, int64_t m, void* lie,
                int64_t ld_lie, const void* x, int64_t ld_x, cudaStream_t s);

// rows idx[i] (or i) of `out` (stride ld) <- the unit tensor
int unit_rows(int mode, void* out, int64_t ld, int64_t cols, const int64_t* idx, int64_t n,
              cudaStream_t s);

// acc[q] <- acc[q] * src[r_0] * src[r_1] * ... with q's source rows
// src_rows[off[q] .. off[q+1]) in order; one gathered product per position,
// ping-ponging between two scratch buffers in factor-count order, and one
// gather back into acc (rows of stride T).  acc_mode RPYB_F64 with src_mode
// RPYB_F32 uses the mixed-precision product.
int ordered_products(int acc_mode, int src_mode, const Geometry& g, int64_t n, void* acc,
                     const void* src, const std::vector<int64_t>& off,
                     const std::vector<int64_t>& src_rows, cudaStream_t s);

// acc[q] <- src[r_0] * src[r_1] * ... (float64; the unit for an empty list),
// or its float64 log when log_out is set (the log's Horner steps run in the
// same block on the product still on the SM), fused: one block per row keeps
// the running product on the SM across its whole list of factors (levels
// below the top in shared memory, the top level in registers).  Available
// for widths 2..6 and 8 when the top level fits the block's registers and
// three copies of its lower levels 200 KB of shared memory.
bool chain_products_available(const Geometry& g);
int chain_products(int src_mode, const Geometry& g, int64_t n, double* acc, const void* src,
                   const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                   bool log_out, cudaStream_t s);
// The same products (float64 accumulation) written straight into rows
// dst_rows[i] of `nodes`, the [*, T] array (of src_mode's type) that also
// holds the factors; the destination rows must not be factors of the call.
// The index lists are copied before the call returns.
int chain_products_into(int src_mode, const Geometry& g, int64_t n, void* nodes,
                        const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                        const std::vector<int64_t>& dst_rows, cudaStream_t s);
// log(product) projected onto the Hall basis inside the chain kernel (the
// log never leaves the SM): Lie coordinates to lie[i * ld_lie + r].  Needs
// the packed t2l map and room for the whole log in shared memory.
bool chain_lie_available(const Geometry& g, const LieMapsDev& maps);
int chain_products_lie(int src_mode, const Geometry& g, int64_t n, const void* src,
                       const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                       const LieMapsDev& maps, double* lie, int64_t ld_lie, cudaStream_t s);

// Bytes of scratch finish_queries needs for up to `n` rows.
size_t finish_scratch_bytes(const Geometry& g, int64_t lie_dim, int64_t n);

// For m group-like float64 rows `acc` ([m, T]; their logs when acc_is_log):
// log-signature t2l(log(acc)) into out_logsig and/or signature
// exp(l2t(logsig)) into out_sig (either may be null).  Scratch from `scratch`.
int finish_queries(const Geometry& g, const LieMapsDev& maps, int64_t m, double* acc,
                   bool acc_is_log, double* out_logsig, int64_t ld_logsig, double* out_sig,
                   int64_t ld_sig, void* scratch, size_t scratch_bytes, cudaStream_t s,
                   bool lie_ready = false);
// Where finish_queries keeps the m rows of Lie coordinates (out_logsig, or
// its scratch), with their stride; lie_ready = true means the caller wrote
// them there already (chain_products_lie) and only out_sig remains.
double* finish_lie_rows(const Geometry& g, int64_t lie_dim, int64_t m, void* scratch,
                        double* out_logsig, int64_t ld_logsig, int64_t* ld_lie);

// Stream::refine_interval (streams/src/stream.cpp:37-71) for a batch of
// clopen queries against a support, then to_dyadic_intervals
// (intervals/src/dyadic_interval.cpp:191-224).  resolution ==
// RPYB_QUERY_RESOLUTION_AUTO picks max(default_resolution,
// query_resolution(length) + 2) per query.  Empty (trimmed-away or zero
// length) queries get no pieces.  Piece i of query q, in [poff[q],
// poff[q+1]), is [k[i], k[i]+1) / 2^p[i].
int refine_and_dissect(int64_t n, const double* inf, const double* sup, double s0, double s1,
                       int32_t default_resolution, int32_t resolution, std::vector<int64_t>& k,
                       std::vector<int32_t>& p, std::vector<int64_t>& poff);

}  // namespace rpyb
