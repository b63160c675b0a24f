// Internal interface of the signature kernels (csrc/signature.cu) used by
// the planner (csrc/signature_plan.cpp).  Not part of the C ABI.
#pragma once

#include "common.cuh"

namespace rpyb {

// Lane shapes G of the specialised kernel for (mode, width, depth), default
// first; false when the shape is served by the generic kernel.
bool signature_lane_shapes(int mode, int width, int depth, int* gs, int* count);

// Lanes per stream of the specialised kernel with lane shape g (-1: none).
int64_t signature_lanes_per_stream(int mode, int width, int depth, int g);

// One launch over n_items work streams (rows offsets[i] .. offsets[i+1]-1);
// item i's signature goes to row dst_row[i] of `out` (>= 0) or row
// ~dst_row[i] of `alt` (< 0), or row i of `out` when dst_row is NULL.
// g_lane = 0 and wpb = 0 take the defaults.  `queue` is device scratch of
// at least 4 bytes.
int signature_launch(int mode, int width, int depth, int g_lane, int wpb, int64_t n_items,
                     const int64_t* offsets, const void* inc, void* out, int64_t ld_out,
                     const int64_t* order, const int64_t* dst_row, void* alt, int64_t ld_alt,
                     int* queue, cudaStream_t s);

// Per-stream error report of float32 signatures `out32` against the float64
// path on the same increments (rpyb_signature_batched's err_out).  ws must
// hold rpyb_signature_batched_workspace_size(RPYB_F32, ..., 1) bytes; its
// first part is not used (it is the float32 launch's workspace).
int signature_error_report(int width, int depth, int64_t n_streams, const int64_t* offsets,
                           const void* inc32, int64_t total_rows, const void* out32,
                           int64_t ld_out, const int64_t* order, double* err_out, void* ws,
                           size_t ws_bytes, cudaStream_t s);

}  // namespace rpyb
