/*
 * rpyb.h -- C ABI of the B200 dense truncated tensor-algebra library
 * (librpyb.so).  Plain C types only: device pointers are `void*`, sizes are
 * int64_t, the CUDA stream is passed as an opaque `void*` (a cudaStream_t;
 * NULL means the legacy default stream).
 *
 * Conventions shared by every entry point
 * ---------------------------------------
 *  - Return value: 0 on success, a negative RPYB_E* code on failure.  The
 *    thread-local message of the last failure is rpyb_last_error().
 *  - The caller owns every buffer.  Device pointers must be device memory
 *    (or managed memory) of the current CUDA device.
 *  - Tensor layout (identical to RoughPy's dense free tensors): degree-major,
 *    level k of a width-d tensor starts at degree_begin[k] = (d^k - 1)/(d - 1);
 *    inside a level, word (a_1 ... a_k) sits at sum_i a_i d^(k-i) (first letter
 *    most significant).  A batch is `batch` rows, row b at base + b*ld.
 *  - dtype: RPYB_F32 (float32 storage; the exact products of float32 words
 *    are accumulated in float64 and rounded once) or RPYB_F64.
 *  - Degree bounds follow roughpy.compute: a max_degree of -1 (or larger than
 *    depth) means `depth`.
 *  - Calls are asynchronous with respect to the host unless stated.  They are
 *    thread-safe and may run concurrently on different streams.
 *  - Entry points that need temporary device memory take (workspace,
 *    workspace_bytes).  Query the size with the matching *_workspace_size
 *    function.  Passing workspace == NULL makes the library take stream-ordered
 *    memory with cudaMallocAsync/cudaFreeAsync on `stream`.
 */
#ifndef RPYB_H
#define RPYB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RPYB_API __attribute__((visibility("default")))
#else
#define RPYB_API
#endif

/* dtypes */
#define RPYB_F32 0
#define RPYB_F64 1

/* status codes */
#define RPYB_OK 0
#define RPYB_E_INVALID (-1)   /* bad argument: shape, dtype, bounds, null pointer */
#define RPYB_E_CUDA (-2)      /* a CUDA runtime call failed */
#define RPYB_E_NOMEM (-3)     /* workspace too small / allocation failed */
#define RPYB_E_TIMEOUT (-4)   /* a bounded device wait ran out */
#define RPYB_E_UNSUPPORTED (-5)

/* Thread-local message describing the most recent failure on this thread. */
RPYB_API const char* rpyb_last_error(void);
/* Library version string. */
RPYB_API const char* rpyb_version(void);
/*
 * Entry points given no workspace take stream-ordered scratch from a
 * library-owned memory pool per device, which keeps freed memory for reuse
 * (repeated calls then map no device memory).  This returns the pooled
 * memory of every device to the driver.  No reference counterpart.
 */
RPYB_API int rpyb_release_cached_memory(void);
/*
 * Bytes of the current device's scratch pool in use by calls in flight and
 * held in reserve (0 and 0 before the first pooled call).  No reference
 * counterpart.
 */
RPYB_API int rpyb_scratch_pool_usage(int64_t* used_bytes, int64_t* reserved_bytes);

/* Number of scalars in a width/depth tensor: (width^(depth+1)-1)/(width-1). */
RPYB_API int64_t rpyb_tensor_size(int32_t width, int32_t depth);

/*
 * out[b] += lhs[b] (x) rhs[b], truncated: the dense free-tensor fused
 * multiply-add over a batch of rows.
 * Replaces: roughpy_compute/dense/basic/free_tensor_fma.hpp:13-53
 *           (rpy::compute::basic::ft_fma), reached from
 *           roughpy/compute/_src/dense_basic.cpp:85-151 (py_dense_ft_fma).
 * deg_bounds = {out_min, out_max, lhs_min, lhs_max, rhs_min, rhs_max}; NULL
 * means {0,-1,0,-1,0,-1}.
 */
RPYB_API int rpyb_ft_fma(int dtype, int32_t width, int32_t depth, int64_t batch,
                         void* out, const void* lhs, const void* rhs,
                         int64_t ld_out, int64_t ld_lhs, int64_t ld_rhs,
                         const int32_t* deg_bounds, void* stream);

/*
 * Row-gathered variant used by tree reductions: for i < n,
 *   out[out_idx[i]] (+)= lhs[lhs_idx[i]] (x) rhs[rhs_idx[i]]
 * with accumulate != 0 selecting += and 0 selecting =.  Index arrays are
 * device int64 arrays; NULL means the identity.  Rows share one ld.
 * No reference counterpart as one call: it batches
 * roughpy_compute/dense/basic/free_tensor_fma.hpp:13-53 over index lists.
 */
RPYB_API int rpyb_ft_mul_gather(int dtype, int32_t width, int32_t depth, int64_t n,
                                void* out, const void* lhs, const void* rhs,
                                int64_t ld, const int64_t* out_idx,
                                const int64_t* lhs_idx, const int64_t* rhs_idx,
                                int accumulate, void* stream);

/*
 * Mixed-precision form of rpyb_ft_mul_gather: float64 output and left rows,
 * float32 right rows, products accumulated in float64.  Used to multiply
 * float32-stored dyadic nodes into float64 query accumulators.  No separate
 * reference counterpart (the reference has no mixed-precision product).
 */
RPYB_API int rpyb_ft_mul_gather_mixed(int32_t width, int32_t depth, int64_t n, double* out,
                                      const double* lhs, const float* rhs, int64_t ld,
                                      const int64_t* out_idx, const int64_t* lhs_idx,
                                      const int64_t* rhs_idx, int accumulate, void* stream);

/*
 * lhs[b] <- lhs[b] (x) rhs[b] in place.
 * Replaces: roughpy_compute/dense/basic/free_tensor_inplace_mul.hpp:13-87,
 *           via roughpy/compute/_src/dense_basic.cpp:193-237.
 * deg_bounds = {lhs_min, lhs_max, rhs_min, rhs_max}; NULL = full.
 */
RPYB_API int64_t rpyb_ft_inplace_mul_workspace_size(int dtype, int32_t width,
                                                    int32_t depth, int64_t batch);
RPYB_API int rpyb_ft_inplace_mul(int dtype, int32_t width, int32_t depth, int64_t batch,
                                 void* lhs, const void* rhs, int64_t ld_lhs,
                                 int64_t ld_rhs, const int32_t* deg_bounds,
                                 void* workspace, size_t workspace_bytes,
                                 void* stream);

/*
 * out[b] <- exp(arg[b]) (level 0 of arg ignored), Horner scheme.
 * Replaces: roughpy_compute/dense/intermediate/free_tensor_exp.hpp:13-37 via
 *           roughpy/compute/_src/dense_intermediate.cpp:62-96.
 * out_depth: -1 = depth.  The reference uses the out bounds for arg too.
 */
RPYB_API int64_t rpyb_ft_exp_workspace_size(int dtype, int32_t width, int32_t depth,
                                            int64_t batch);
RPYB_API int rpyb_ft_exp(int dtype, int32_t width, int32_t depth, int64_t batch,
                         void* out, const void* arg, int64_t ld_out, int64_t ld_arg,
                         int32_t out_depth, void* workspace, size_t workspace_bytes,
                         void* stream);

/*
 * rpyb_ft_exp without any device allocation, for callers that cannot call
 * cudaMalloc (a host application that owns every device allocation through a
 * fixed pool, a thread where an allocation would synchronise the device, a
 * callback that forbids allocation).  No counterpart in the reference: it is
 * rpyb_ft_exp with its scratch taken from a file-scope device array of
 * rpyb_ft_exp_noalloc_max_bytes() bytes (8 MiB) that every GPU loading the
 * library holds until exit.  Calls needing more (batch * tensor_size *
 * element size) fail with RPYB_E_INVALID.  The first call on a device looks
 * up the array's device address; make it before any stream capture.  The
 * address is kept for the life of the process: do not reset the device
 * (cudaDeviceReset) between calls, which would reload the module elsewhere.
 * All calls on a device share the array, so calls that overlap on the GPU
 * race: order them on one stream or with events.
 */
RPYB_API int64_t rpyb_ft_exp_noalloc_max_bytes(void);
RPYB_API int rpyb_ft_exp_noalloc(int dtype, int32_t width, int32_t depth, int64_t batch,
                                 void* out, const void* arg, int64_t ld_out, int64_t ld_arg,
                                 int32_t out_depth, void* stream);

/*
 * out[b] <- multiplier[b] * exp(exponent[b]) (level 0 of exponent ignored).
 * Replaces: roughpy_compute/dense/intermediate/free_tensor_fmexp.hpp:15-40 via
 *           roughpy/compute/_src/dense_intermediate.cpp:127-196.
 */
RPYB_API int64_t rpyb_ft_fmexp_workspace_size(int dtype, int32_t width,
                                              int32_t depth, int64_t batch);
RPYB_API int rpyb_ft_fmexp(int dtype, int32_t width, int32_t depth, int64_t batch,
                           void* out, const void* multiplier, const void* exponent,
                           int64_t ld_out, int64_t ld_mul, int64_t ld_exp,
                           int32_t out_depth, void* workspace,
                           size_t workspace_bytes, void* stream);

/*
 * out[b] <- log(arg[b]), assuming arg level 0 == 1 (it is masked).  The
 * series is always evaluated in float64 on the device (float32 rows are
 * widened), because its alternating terms cancel.  As in the reference, the
 * incoming out[b][0] is added to the first Horner coefficient (pass zeroed
 * rows for the plain logarithm).
 * Replaces: roughpy_compute/dense/intermediate/free_tensor_log.hpp:12-39 via
 *           roughpy/compute/_src/dense_intermediate.cpp:204-294.
 */
RPYB_API int64_t rpyb_ft_log_workspace_size(int dtype, int32_t width, int32_t depth,
                                            int64_t batch);
RPYB_API int rpyb_ft_log(int dtype, int32_t width, int32_t depth, int64_t batch,
                         void* out, const void* arg, int64_t ld_out, int64_t ld_arg,
                         int32_t out_depth, int32_t arg_depth, void* workspace,
                         size_t workspace_bytes, void* stream);

/*
 * out[b] <- antipode(arg[b]): word reversal with sign (-1)^degree.
 * Replaces: roughpy_compute/dense/basic/free_tensor_antipode.hpp:50-100 via
 *           roughpy/compute/_src/dense_basic.cpp:244-330.
 */
RPYB_API int rpyb_ft_antipode(int dtype, int32_t width, int32_t depth, int64_t batch,
                              void* out, const void* arg, int64_t ld_out,
                              int64_t ld_arg, void* stream);

/*
 * out[b] += L*_{op[b]}(arg[b]): adjoint of left free-tensor multiplication
 * (acts on shuffle tensors).  deg = {out_depth, op_depth, arg_depth} (-1 = depth).
 * Replaces: roughpy_compute/dense/basic/free_tensor_adjoint_left_mul.hpp:11-77
 *           via roughpy/compute/_src/dense_basic.cpp (py_dense_ft_adj_lmul).
 */
RPYB_API int rpyb_ft_adjoint_left_mul(int dtype, int32_t width, int32_t depth,
                                      int64_t batch, void* out, const void* op,
                                      const void* arg, int64_t ld_out, int64_t ld_op,
                                      int64_t ld_arg, const int32_t* deg,
                                      void* stream);

/*
 * Batched path signatures: for each stream s, with increments rows
 * offsets[s] .. offsets[s+1]-1 of `increments` ([total, width] row-major),
 *   out[s] = exp(x_0) (x) exp(x_1) (x) ... (x) exp(x_{L-1})   (Chen product)
 * mode RPYB_F64: float64 increments/output, plain float64 arithmetic.
 * mode RPYB_F32: float32 increments/output, float32 products with lazily
 *   compensated (two-sum folded) accumulation of the running signature.
 * One persistent launch; work items are taken longest-stream first from a
 * device-side queue.  `order` (device int64[n_streams], nullable) gives the
 * processing order (longest first is best); `offsets` is a device int64
 * array of n_streams+1 entries.  An empty stream gives the unit tensor.
 * Replaces: algebra/src/lite_context.h:542-563 (compute_signature: a chain of
 *           fmexp over increments) and the reference recipe of chaining
 *           roughpy_compute/dense/intermediate/free_tensor_fmexp.hpp:15-40.
 */
RPYB_API int64_t rpyb_signature_workspace_size(int mode, int32_t width, int32_t depth,
                                               int64_t n_streams);
RPYB_API int rpyb_signature(int mode, int32_t width, int32_t depth, int64_t n_streams,
                            const int64_t* offsets, const void* increments,
                            void* out, int64_t ld_out, const int64_t* order,
                            void* workspace, size_t workspace_bytes, void* stream);

/*
 * rpyb_signature with an accuracy report.  err_out (device float64
 * [n_streams], nullable) receives, per stream, the largest per-level relative
 * error max_k ||out_k - ref_k||_inf / ||ref_k||_inf of the result against the
 * float64 GPU path run on the same increments in the same launch layout (the
 * absolute error for a level whose reference is zero).  For RPYB_F64 the
 * result is its own reference and err_out is zeroed.  total_rows =
 * offsets[n_streams] (the host value; it sizes the float64 copy of the
 * increments).  The report costs one float64 launch besides the float32 one;
 * its workspace holds the float64 signatures ([n_streams, tensor_size]) and
 * increments.  err_out == NULL is rpyb_signature.
 * Replaces: the same reference path as rpyb_signature; the report is the
 * per-result accuracy statement of the float32 mode (the reference computes
 * in float64 only).
 */
RPYB_API int64_t rpyb_signature_batched_workspace_size(int mode, int32_t width, int32_t depth,
                                                       int64_t n_streams, int64_t total_rows,
                                                       int with_error);
RPYB_API int rpyb_signature_batched(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                    const int64_t* offsets, const void* increments,
                                    int64_t total_rows, void* out, int64_t ld_out,
                                    const int64_t* order, double* err_out, void* workspace,
                                    size_t workspace_bytes, void* stream);

/*
 * Signature plans: a batch layout whose stream lengths are known on the host
 * (offsets_host, n_streams + 1 entries), with its launch schedule and device
 * tables, reused across calls.  A schedule sets the kernel's lane shape (the
 * level split: level-(N-1) words per lane), the warps per block and a time-
 * segment length: streams longer than it are cut into balanced segments that
 * run as separate work items of the persistent launch, and the segment
 * signatures are multiplied back in order by a pairwise tree of batched
 * products (the Chen product is associative), so a few very long streams
 * still fill the GPU.  The schedule comes from RPYB_SIG_SCHEDULE
 * ("g=8,wpb=0,seg=4096"), else from the JSON cache at RPYB_SIG_TUNE_CACHE
 * (default $XDG_CACHE_HOME/roughpy_b200/signature_schedules.json) keyed on
 * (device, mode, width, depth, log2 longest stream, log2 batch size), else,
 * with flags & RPYB_SIG_PLAN_TUNE, by timing the candidates on synthetic
 * increments of this layout on `stream` (then cached); otherwise the
 * defaults.  Creation allocates the plan's device memory and waits for
 * `stream`; rpyb_sig_plan_run allocates nothing (except the float64 buffers
 * of the first call with err_out, see rpyb_signature_batched).  One run at a
 * time per plan.  rpyb_sig_plan_describe writes a JSON description of the
 * schedule into buf (cap bytes) and returns its length.
 * Replaces: algebra/src/lite_context.h:542-563 (compute_signature) for a
 *           batch, like rpyb_signature.
 */
typedef struct rpyb_sig_plan rpyb_sig_plan;
#define RPYB_SIG_PLAN_TUNE 1
RPYB_API int rpyb_sig_plan_create(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                  const int64_t* offsets_host, int32_t flags, void* stream,
                                  rpyb_sig_plan** plan);
RPYB_API int rpyb_sig_plan_run(rpyb_sig_plan* plan, const void* increments, void* out,
                               int64_t ld_out, double* err_out, void* stream);
RPYB_API int rpyb_sig_plan_describe(const rpyb_sig_plan* plan, char* buf, int64_t cap);
RPYB_API int rpyb_sig_plan_free(rpyb_sig_plan* plan);

/*
 * rpyb_signature from host memory, end to end: increments [total, width] and
 * the output [n_streams, ld_out] are HOST buffers (pin them for overlap),
 * offsets_host is a host int64 array.  The streams are processed in n_chunks
 * contiguous groups of about equal total length; the host->device copy of
 * chunk i+1 and the device->host copy of chunk i-1 overlap the kernel of
 * chunk i (two internal copy streams, double-buffered device chunks in
 * device_buffer, sized by rpyb_signature_host_device_bytes; NULL = stream-
 * ordered allocation).  Completion is ordered on `stream`: synchronise it
 * before reading out_host.
 * Replaces: the same reference path as rpyb_signature, called with host data.
 */
RPYB_API int64_t rpyb_signature_host_device_bytes(int mode, int32_t width, int32_t depth,
                                                  int64_t n_streams, const int64_t* offsets_host,
                                                  int32_t n_chunks);
RPYB_API int rpyb_signature_host(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                 const int64_t* offsets_host, const void* inc_host,
                                 void* out_host, int64_t ld_out, int32_t n_chunks,
                                 void* device_buffer, size_t device_bytes, void* stream);

/*
 * Reverse-mode derivative of rpyb_signature: given the upstream gradient
 * grad_sig (dLoss/dS per stream, [n_streams, T] with row stride ld_grad, or
 * one shared row when ld_grad == 0), writes grad_inc = dLoss/d increments
 * ([total, width]).  One block per stream walks it backwards, propagating
 * the adjoint G_t = exp(D_x) G_{t+1} (the reverse Chen product) and the
 * increment gradients; states are recovered by inverse steps re-anchored on
 * float64 checkpoints every `checkpoint_every` steps (widths 2..8 with
 * width^(depth-2) <= 992), or recomputed per segment from them (other
 * shapes).  Adjoint accumulators are float64 in both modes.  `max_len` sizes
 * the checkpoint scratch and must bound every stream length; -1 takes the
 * longest stream.  Before launching, the call reduces the offsets on the
 * device and reads the longest and shortest length back (a 16-byte read that
 * waits for `stream`; the call is therefore not capturable in a CUDA graph):
 * a stream longer than max_len, or decreasing offsets, fail with
 * RPYB_E_INVALID and nothing is written.  Width <= 8.
 * No reference counterpart: RoughPy only has the forward-mode derivative
 * (algebra/src/lite_context.h:577-636, LiteContext::sig_derivative_impl).
 */
RPYB_API int64_t rpyb_signature_backward_workspace_size(int mode, int32_t width, int32_t depth,
                                                        int64_t n_streams, int64_t max_len,
                                                        int32_t checkpoint_every);
RPYB_API int rpyb_signature_backward(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                     const int64_t* offsets, int64_t max_len,
                                     const void* increments, const void* grad_sig,
                                     int64_t ld_grad, void* grad_inc, int32_t checkpoint_every,
                                     void* workspace, size_t workspace_bytes, void* stream);

/*
 * Lie basis (Hall set) and the Lie <-> tensor maps, built on the host.
 * rpyb_lie_basis_size: number of Hall keys of degree 1..depth (excludes the
 * null key 0).  rpyb_lie_basis_data fills data[(size+1)*2] (parent pairs,
 * row 0 = (0,0)) and degree_begin[depth+2], identical to
 * roughpy/compute/_src/lie_basis.c:201-337 (construct_lie_basis).
 */
RPYB_API int64_t rpyb_lie_basis_size(int32_t width, int32_t depth);
RPYB_API int rpyb_lie_basis_data(int32_t width, int32_t depth, int64_t* data,
                                 int64_t* degree_begin);
/*
 * CSR form of the maps.  which = 0: l2t (tensor_size rows x lie_size cols),
 * which = 1: t2l (lie_size rows x tensor_size cols, rbracketing / degree).
 * Call with indices == NULL to get the number of stored entries (return
 * value >= 0), then again with arrays of that size.  Values in float64.
 * Replaces: roughpy/compute/_src/lie_basis.c:902-950 (l2t) and :1066-1200
 *           (t2l), vendored/libalgebra_lite/include/libalgebra_lite/maps.h:131-210.
 */
RPYB_API int64_t rpyb_lie_map_csr(int32_t width, int32_t depth, int which,
                                  int64_t* indptr, int64_t* indices, double* values);

/*
 * y[b] += scale * M x[b] for a CSR matrix M (device arrays, float64 values),
 * batched over rows; x, y of dtype (float32 rows are computed in float64).
 * The map accumulates into y, as the reference's does: zero y for a plain
 * product.  Entries whose column index lies outside [0, n_cols) are skipped.
 * Replaces: roughpy_compute/dense/basic/apply_sparse_linear_map.hpp:16-55 via
 *           roughpy/compute/_src/dense_basic.cpp:564-620 and :1055-1150.
 */
RPYB_API int rpyb_sparse_map(int dtype, int64_t n_rows, int64_t n_cols, int64_t batch,
                             const int64_t* indptr, const int64_t* indices,
                             const double* values, void* y, const void* x,
                             int64_t ld_y, int64_t ld_x, double scale, void* stream);

/*
 * Batched tensor -> Lie (Hall coordinates, rbracketing / degree) and
 * Lie -> tensor maps with the maps kept on the device (uploaded once per
 * device and shape).  Both assign their output rows.
 * Replaces: roughpy/compute/_src/dense_basic.cpp:1055-1150
 *           (py_dense_tensor_to_lie) and :564-620 (py_dense_lie_to_tensor),
 *           i.e. Context::tensor_to_lie / lie_to_tensor
 *           (algebra/include/roughpy/algebra/context.h:171-172).
 */
RPYB_API int rpyb_tensor_to_lie(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                                int64_t ld_out, const void* arg, int64_t ld_arg, void* stream);
RPYB_API int rpyb_lie_to_tensor(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                                int64_t ld_out, const void* arg, int64_t ld_arg, void* stream);

/*
 * Dissection of the clopen interval [inf, sup) into maximal dyadic pieces at
 * resolution `tol`, in order.  Piece i is [k[i] / 2^p[i], (k[i]+1) / 2^p[i]).
 * Writes at most `cap` pieces and returns the number of pieces (which may
 * exceed cap), or a negative status.  Opencl intervals are rejected, as the
 * reference does not implement them either.
 * Replaces: intervals/src/dyadic_interval.cpp:191-224 (to_dyadic_intervals).
 */
RPYB_API int64_t rpyb_dyadic_dissect(double inf, double sup, int32_t tol, int clopen,
                                     int64_t* k, int32_t* p, int64_t cap);
/* Batched form: query q's pieces are written to [offsets[q], offsets[q+1]). */
RPYB_API int rpyb_dyadic_dissect_batch(int64_t n, const double* inf, const double* sup,
                                       const int32_t* tol, int clopen, int64_t* k,
                                       int32_t* p, int64_t cap, int64_t* offsets);

/*
 * Dyadic signature tree of a stream of Lie increments (opaque, device-
 * resident), and batched interval queries against it.
 *
 * rpyb_dyadic_build: events e < n_events at non-decreasing times_host[e]
 * (host array) carry device rows `rows` ([n_events, row_len], float64 for
 * RPYB_F64, float32 for RPYB_F32): level-1 increments (row_len == width) or
 * Hall-basis Lie coordinates (row_len == rpyb_lie_basis_size).  Leaves are the
 * dyadic intervals of `resolution` meeting the support [support_inf,
 * support_sup) and the event times; each leaf is the Chen product of exp over
 * its events, and every coarser aligned dyadic block is the product of its
 * halves.  The handle owns its device memory (allocated on the current
 * device, released by rpyb_dyadic_free); the build is ordered on `stream`.
 * Replaces: the LieIncrementStream constructor and the DyadicCachingLayer
 * cache (streams/src/lie_increment_stream.cpp:116-199,
 * streams/src/dyadic_caching_layer.cpp:86-154), which cache leaves only and
 * recompute coarser pieces by recursive CBH.
 *
 * rpyb_dyadic_query: for each clopen query [inf_host[q], sup_host[q]) (host
 * arrays; inf <= sup), trims to the support, dissects at `resolution`
 * (RPYB_QUERY_RESOLUTION_AUTO: the reference's per-query choice
 * max(stream resolution, query_resolution(length) + 2)), multiplies the
 * pieces' node signatures in order in float64 and writes the log-signature
 * in Hall coordinates (out_logsig, [n, ld_logsig], device float64) and/or
 * the signature exp(l2t(logsig)) (out_sig, [n, ld_sig]); either may be NULL.
 * Thread-safe on a built tree; temporaries are stream-ordered allocations.
 * Replaces: Stream::log_signature / Stream::signature
 * (streams/src/stream.cpp:54-171) with intervals/src/dyadic_interval.cpp:191-224
 * and algebra/src/context.cpp:156-215.
 *
 * rpyb_dyadic_tree_info / rpyb_dyadic_node_row expose the node table (rows of
 * tensor_size values of the mode's type) for inspection; node_row returns the
 * row of dyadic block `block` at `level` levels above the leaves (the
 * interval [block, block+1) * 2^(level - resolution)), or -1.
 */
typedef struct rpyb_dyadic_tree rpyb_dyadic_tree;
/*
 * rpyb_dyadic_save / rpyb_dyadic_load: a built tree as one host byte block
 * (a fixed header with the tensor shape, mode, resolution and support, the
 * per-level block tables, then the node table of the mode's type) and back,
 * so that a stream's cached signatures outlive the process or move to
 * another device.  save copies the node table to the host and waits for
 * `stream`; it returns the bytes written (rpyb_dyadic_save_size) or a
 * negative status.  load validates the block, allocates the nodes on the
 * current device and copies them there (waiting for `stream`); the loaded
 * tree answers rpyb_dyadic_query exactly as the saved one.
 * Replaces: DyadicCachingLayer::dump_cache / load_cache
 *           (streams/src/dyadic_caching_layer.cpp:168-201), which write the
 *           resolution-level Lie cache through cereal; here the whole tree
 *           is saved, so nothing is recomputed after loading.
 */
RPYB_API int64_t rpyb_dyadic_save_size(const rpyb_dyadic_tree* tree);
RPYB_API int64_t rpyb_dyadic_save(const rpyb_dyadic_tree* tree, void* buf, int64_t cap,
                                  void* stream);
RPYB_API int rpyb_dyadic_load(const void* buf, int64_t size, rpyb_dyadic_tree** tree,
                              void* stream);
#define RPYB_QUERY_RESOLUTION_AUTO (-2147483647 - 1)
RPYB_API int rpyb_dyadic_build(int mode, int32_t width, int32_t depth, int32_t resolution,
                               double support_inf, double support_sup, int64_t n_events,
                               const double* times_host, const void* rows, int32_t row_len,
                               rpyb_dyadic_tree** tree, void* stream);
RPYB_API int rpyb_dyadic_free(rpyb_dyadic_tree* tree);
/*
 * Range-product table of a tree: with blocks of 2^block_log2 leaves (0 picks
 * about the square root of the leaf count), the product of the leaves from
 * each leaf to its block's ends (both ways) and a disjoint sparse table over
 * the blocks, computed in float64 and stored in the tree's type.  A later
 * rpyb_dyadic_query whose pieces are no finer than the leaves and span more
 * than one block then multiplies at most four table rows instead of every
 * piece (the same product, associated differently).  The table doubles the
 * tree's device memory; trees of fewer than four blocks get none.  Waits for
 * `stream`.  No reference counterpart: the reference recomputes coarse
 * pieces recursively (streams/src/dyadic_caching_layer.cpp:86-154).
 */
RPYB_API int rpyb_dyadic_range_table(rpyb_dyadic_tree* tree, int32_t block_log2, void* stream);
RPYB_API int rpyb_dyadic_tree_info(const rpyb_dyadic_tree* tree, int64_t* rows,
                                   int32_t* top_level, const void** nodes);
RPYB_API int64_t rpyb_dyadic_node_row(const rpyb_dyadic_tree* tree, int32_t level,
                                      int64_t block);
RPYB_API int rpyb_dyadic_query(const rpyb_dyadic_tree* tree, int64_t n_queries,
                               const double* inf_host, const double* sup_host,
                               int32_t resolution, double* out_logsig, int64_t ld_logsig,
                               double* out_sig, int64_t ld_sig, void* stream);

/*
 * Log-signatures / signatures of clopen intervals of a piecewise abelian
 * stream: pieces j < n_pieces are [piece_inf[j], piece_sup[j]) (host arrays,
 * in order) carrying Lie elements piece_lies ([n_pieces, ld_lies] device
 * float64 Hall coordinates).  Each query is trimmed to [support_inf,
 * support_sup), dissected at `resolution` (RPYB_QUERY_RESOLUTION_AUTO: the
 * reference's per-query choice from default_resolution), and each dyadic
 * interval [a, b) collects the pieces meeting it: whole when inside, else
 * scaled by (sup_j - a) / (sup_j - inf_j) as the reference does; all
 * contributions are combined by CBH (the log of the ordered product of their
 * exponentials, in float64).  Outputs as rpyb_dyadic_query.
 * Replaces: streams/src/piecewise_abelian_stream.cpp:154-189 through
 *           streams/src/stream_base.cpp:81-96 and streams/src/stream.cpp:54-171.
 */
RPYB_API int rpyb_piecewise_query(int32_t width, int32_t depth, int64_t n_pieces,
                                  const double* piece_inf, const double* piece_sup,
                                  const double* piece_lies, int64_t ld_lies, double support_inf,
                                  double support_sup, int32_t default_resolution,
                                  int64_t n_queries, const double* inf_host,
                                  const double* sup_host, int32_t resolution, double* out_logsig,
                                  int64_t ld_logsig, double* out_sig, int64_t ld_sig,
                                  void* stream);

/*
 * Batched Campbell-Baker-Hausdorff products: for each list q, with items
 * i in [offsets_host[q], offsets_host[q+1]) of `lies` (device float64
 * [items, ld_lies] Hall coordinates),
 *   out[q] = t2l(log(exp(l2t(x_first)) ... exp(l2t(x_last))))
 * in float64 (device [n_lists, ld_out]).  A one-element list returns its
 * element, an empty list zero, as the reference does.  Temporaries are
 * stream-ordered allocations; the call waits for `stream` when a list has a
 * single element (the host index table of that copy must outlive it).
 * Replaces: Context::cbh (algebra/src/context.cpp:187-208), one list per call
 *           in the reference.
 */
RPYB_API int rpyb_cbh(int32_t width, int32_t depth, int64_t n_lists, const int64_t* offsets_host,
                      const double* lies, int64_t ld_lies, double* out, int64_t ld_out,
                      void* stream);

/*
 * Forward-mode derivative of signatures along Lie perturbations, batched over
 * independent lists.  List q holds the pairs i in [offsets_host[q],
 * offsets_host[q+1]) of rows of `logsig` (the log-signature of an interval)
 * and `perturbation`, both Hall-basis Lie coordinates ([items, ld_lie] device
 * arrays of dtype).  With X = l2t(logsig_i), P = l2t(perturbation_i):
 *   out[q] = 0;  out[q] <- out[q] * exp(X) + exp(X) * sum_k (-1)^k ad_X^k(P) / (k+1)!
 * over the list in order, exactly as the reference states it; for one pair
 * this is the directional derivative of exp at X along P.  Scratch from
 * `workspace` (rpyb_sig_derivative_workspace_size) or, when NULL, stream-
 * ordered allocation.
 * Replaces: algebra/src/lite_context.h:577-636 (LiteContext::sig_derivative_impl,
 *           derive_series_compute, sig_derivative_single), reached from
 *           Stream::signature_derivative (streams/src/stream.cpp:173-230).
 */
RPYB_API int64_t rpyb_sig_derivative_workspace_size(int dtype, int32_t width, int32_t depth,
                                                    int64_t n_lists, int64_t n_items);
RPYB_API int rpyb_sig_derivative(int dtype, int32_t width, int32_t depth, int64_t n_lists,
                                 const int64_t* offsets_host, const void* logsig,
                                 const void* perturbation, int64_t ld_lie, void* out,
                                 int64_t ld_out, void* workspace, size_t workspace_bytes,
                                 void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RPYB_H */
