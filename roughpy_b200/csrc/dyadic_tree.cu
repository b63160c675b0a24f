// Dyadic signature tree of a stream of Lie increments, and batched interval
// queries against it: the native runtime behind LieIncrementStream's
// signature / log_signature.
//
// The reference keeps a std::map<DyadicInterval, Lie> cache at the stream
// resolution only and recomputes every coarser piece by recursive CBH of its
// halves (streams/src/dyadic_caching_layer.cpp:86-154), one query at a time
// on the host.  Here the whole tree lives on the device as dense tensors:
//
//   * leaves = the dyadic intervals of the stream resolution R that meet the
//     support; leaf i is the Chen product of exp(event) over the events it
//     contains (the batched signature kernel for level-1 increments, or
//     exp(l2t(lie)) and ordered products for Hall coordinates);
//   * level j holds the aligned blocks of 2^j leaves, node = left * right
//     (one gathered batched product launch per level).  Block ranges follow
//     floor division, so a support on both sides of 0 works: merging stops
//     at the pair of blocks -1, 0 (no dyadic interval spans the origin).
//
// A query [a, b) is trimmed to the support (streams/src/stream.cpp:37-71),
// dissected into maximal dyadic pieces on the host
// (intervals/src/dyadic_interval.cpp:191-224), each piece is mapped to a tree
// node, and every query's node signatures are multiplied in order on the
// device in float64 (float32 nodes enter through the mixed-precision
// product).  log, then the tensor->Lie map, give the log-signature
// (algebra/src/context.cpp:156-215); the signature is exp(l2t(logsig)).
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "common.cuh"

struct rpyb_dyadic_tree {
    int mode = 0;
    int32_t width = 0, depth = 0, resolution = 0;
    double s0 = 0.0, s1 = 0.0;
    int device = 0;
    rpyb::Geometry g;
    int J = 0;                              // top level
    std::vector<int64_t> lo, cnt, base;     // per level: first block, blocks, first row
    int64_t unit_row = 0, rows = 0;
    void* nodes = nullptr;                  // [rows, T] of the mode's type
    int64_t lie_dim = 0;
    // Lie maps (CSR, float64 values) on the device
    int64_t* t2l_ptr = nullptr;
    int64_t* t2l_idx = nullptr;
    double* t2l_val = nullptr;
    int64_t* l2t_ptr = nullptr;
    int64_t* l2t_idx = nullptr;
    double* l2t_val = nullptr;
};

namespace rpyb {
namespace {

// rows[idx[i]] <- unit (1 at word 0, 0 elsewhere)
template <typename T>
__global__ void unit_rows_kernel(T* __restrict__ out, int64_t ld, int64_t cols,
                                 const int64_t* __restrict__ idx, int64_t n)
{
    const int64_t total = n * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / cols, c = e - i * cols;
        const int64_t r = idx ? idx[i] : i;
        out[r * ld + c] = (c == 0) ? T(1) : T(0);
    }
}

// dst[idx[i]] <- src[i] for i < n (rows of `cols` values)
template <typename T>
__global__ void scatter_rows_kernel(T* __restrict__ dst, int64_t ld_dst, const T* __restrict__ src,
                                    int64_t ld_src, int64_t cols, const int64_t* __restrict__ idx,
                                    int64_t n)
{
    const int64_t total = n * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / cols, c = e - i * cols;
        dst[idx[i] * ld_dst + c] = src[i * ld_src + c];
    }
}

unsigned grid_for(int64_t total)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
}

template <typename T>
int unit_rows(T* out, int64_t ld, int64_t cols, const int64_t* idx, int64_t n, cudaStream_t s)
{
    if (n <= 0) return RPYB_OK;
    unit_rows_kernel<T><<<grid_for(n * cols), 256, 0, s>>>(out, ld, cols, idx, n);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

template <typename T>
int scatter_rows(T* dst, int64_t ld_dst, const T* src, int64_t ld_src, int64_t cols,
                 const int64_t* idx, int64_t n, cudaStream_t s)
{
    if (n <= 0) return RPYB_OK;
    scatter_rows_kernel<T><<<grid_for(n * cols), 256, 0, s>>>(dst, ld_dst, src, ld_src, cols, idx, n);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

// acc[q] <- acc[q] * src[r_0] * src[r_1] * ... with q's source rows
// src_rows[off[q] .. off[q+1]) in order; one gathered product per position.
// acc_mode: RPYB_F64 or RPYB_F32; a float64 accumulator over float32 sources
// uses the mixed-precision product.  acc rows have stride T, src rows T.
int ordered_products(int acc_mode, int src_mode, const Geometry& g, int64_t n, void* acc,
                     const void* src, const std::vector<int64_t>& off,
                     const std::vector<int64_t>& src_rows, cudaStream_t s)
{
    const int64_t T = g.size();
    int64_t maxc = 0;
    for (int64_t q = 0; q < n; ++q) maxc = std::max(maxc, off[q + 1] - off[q]);
    if (n == 0 || maxc == 0) return RPYB_OK;
    const bool mixed = acc_mode == RPYB_F64 && src_mode == RPYB_F32;
    if (!mixed && acc_mode != src_mode) return fail(RPYB_E_INVALID, "unsupported dtype pair");
    const int64_t es = acc_mode == RPYB_F64 ? 8 : 4;
    // host index lists for every position, uploaded in one copy:
    // position r uses q_idx[pos[r] .. pos[r+1]) and node[pos[r] .. pos[r+1])
    std::vector<int64_t> pos(maxc + 1, 0), packed;
    packed.reserve(2 * (size_t)off[n]);
    int64_t max_active = 0;
    for (int64_t r = 0; r < maxc; ++r) {
        pos[r] = (int64_t)packed.size() / 2;
        std::vector<int64_t> qs, ns;
        for (int64_t q = 0; q < n; ++q)
            if (off[q + 1] - off[q] > r) {
                qs.push_back(q);
                ns.push_back(src_rows[off[q] + r]);
            }
        max_active = std::max<int64_t>(max_active, (int64_t)qs.size());
        // interleave as two consecutive blocks per position
        packed.insert(packed.end(), qs.begin(), qs.end());
        packed.insert(packed.end(), ns.begin(), ns.end());
    }
    pos[maxc] = (int64_t)packed.size() / 2;
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    const size_t idx_bytes = (packed.size() * 8 + 255) / 256 * 256;
    int rc;
    if ((rc = sc.get(idx_bytes + (size_t)(max_active * T * es), &mem))) return rc;
    int64_t* d_idx = static_cast<int64_t*>(mem);
    void* tmp = static_cast<char*>(mem) + idx_bytes;
    RPYB_CUDA(cudaMemcpyAsync(d_idx, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice, s));
    for (int64_t r = 0; r < maxc; ++r) {
        const int64_t m = pos[r + 1] - pos[r];
        const int64_t* q_idx = d_idx + 2 * pos[r];
        const int64_t* n_idx = q_idx + m;
        if (mixed)
            rc = rpyb_ft_mul_gather_mixed(g.width, g.depth, m, static_cast<double*>(tmp),
                                          static_cast<const double*>(acc),
                                          static_cast<const float*>(src), T, nullptr, q_idx,
                                          n_idx, 0, s);
        else
            rc = rpyb_ft_mul_gather(acc_mode, g.width, g.depth, m, tmp, acc, src, T, nullptr,
                                    q_idx, n_idx, 0, s);
        if (rc) return rc;
        if (acc_mode == RPYB_F64)
            rc = scatter_rows(static_cast<double*>(acc), T, static_cast<const double*>(tmp), T, T,
                              q_idx, m, s);
        else
            rc = scatter_rows(static_cast<float*>(acc), T, static_cast<const float*>(tmp), T, T,
                              q_idx, m, s);
        if (rc) return rc;
    }
    // the packed host vector is read by the copy before cudaMemcpyAsync
    // returns (pageable source), so it may go out of scope here
    return RPYB_OK;
}

int upload_map(int32_t w, int32_t d, int which, int64_t n_rows, int64_t** ptr, int64_t** idx,
               double** val)
{
    const int64_t nnz = rpyb_lie_map_csr(w, d, which, nullptr, nullptr, nullptr);
    if (nnz < 0) return (int)nnz;
    std::vector<int64_t> hp(n_rows + 1), hi(std::max<int64_t>(nnz, 1));
    std::vector<double> hv(std::max<int64_t>(nnz, 1));
    const int64_t got = rpyb_lie_map_csr(w, d, which, hp.data(), hi.data(), hv.data());
    if (got < 0) return (int)got;
    RPYB_CUDA(cudaMalloc(ptr, hp.size() * 8));
    RPYB_CUDA(cudaMalloc(idx, hi.size() * 8));
    RPYB_CUDA(cudaMalloc(val, hv.size() * 8));
    RPYB_CUDA(cudaMemcpy(*ptr, hp.data(), hp.size() * 8, cudaMemcpyHostToDevice));
    RPYB_CUDA(cudaMemcpy(*idx, hi.data(), hi.size() * 8, cudaMemcpyHostToDevice));
    RPYB_CUDA(cudaMemcpy(*val, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice));
    return RPYB_OK;
}

void release(rpyb_dyadic_tree* t)
{
    if (!t) return;
    int cur = 0;
    const bool switched = cudaGetDevice(&cur) == cudaSuccess && cur != t->device &&
                          cudaSetDevice(t->device) == cudaSuccess;
    for (void* p : {(void*)t->nodes, (void*)t->t2l_ptr, (void*)t->t2l_idx, (void*)t->t2l_val,
                    (void*)t->l2t_ptr, (void*)t->l2t_idx, (void*)t->l2t_val})
        if (p) cudaFree(p);
    if (switched) cudaSetDevice(cur);
    delete t;
}

// streams/include/roughpy/streams/stream_base.h:74-83 (query_resolution)
int32_t query_param_to_resolution(double length)
{
    int e = 0;
    std::frexp(length, &e);
    return -std::min(0, e - 1);
}

int64_t node_row(const rpyb_dyadic_tree* t, int64_t level, int64_t blk)
{
    if (level < 0 || level > t->J) return -1;
    const int64_t rel = blk - t->lo[level];
    if (rel < 0 || rel >= t->cnt[level]) return -1;
    return t->base[level] + rel;
}

int build_levels(rpyb_dyadic_tree* t, cudaStream_t s)
{
    const Geometry& g = t->g;
    std::vector<int64_t> packed, start(t->J + 2, 0);
    for (int j = 1; j <= t->J; ++j) {
        start[j] = (int64_t)packed.size();
        const int64_t n = t->cnt[j];
        std::vector<int64_t> o(n), l(n), r(n);
        for (int64_t i = 0; i < n; ++i) {
            const int64_t b = t->lo[j] + i;
            o[i] = t->base[j] + i;
            const int64_t c0 = 2 * b, c1 = 2 * b + 1;
            auto row = [&](int64_t c) {
                const int64_t rel = c - t->lo[j - 1];
                return (rel >= 0 && rel < t->cnt[j - 1]) ? t->base[j - 1] + rel : t->unit_row;
            };
            l[i] = row(c0);
            r[i] = row(c1);
        }
        packed.insert(packed.end(), o.begin(), o.end());
        packed.insert(packed.end(), l.begin(), l.end());
        packed.insert(packed.end(), r.begin(), r.end());
    }
    if (packed.empty()) return RPYB_OK;
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    int rc;
    if ((rc = sc.get(packed.size() * 8, &mem))) return rc;
    int64_t* d = static_cast<int64_t*>(mem);
    RPYB_CUDA(cudaMemcpyAsync(d, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice, s));
    for (int j = 1; j <= t->J; ++j) {
        const int64_t n = t->cnt[j];
        const int64_t* o = d + start[j];
        if ((rc = rpyb_ft_mul_gather(t->mode, g.width, g.depth, n, t->nodes, t->nodes, t->nodes,
                                     g.size(), o, o + n, o + 2 * n, 0, s)))
            return rc;
    }
    return RPYB_OK;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int rpyb_dyadic_build(int mode, int32_t width, int32_t depth, int32_t resolution,
                               double support_inf, double support_sup, int64_t n_events,
                               const double* times_host, const void* rows, int32_t row_len,
                               rpyb_dyadic_tree** out_tree, void* stream)
{
    int rc;
    if (!out_tree) return fail(RPYB_E_INVALID, "null tree handle");
    *out_tree = nullptr;
    if (mode != RPYB_F32 && mode != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported mode");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (resolution < -60 || resolution > 60) return fail(RPYB_E_INVALID, "resolution out of range");
    if (!(support_inf <= support_sup) || !std::isfinite(support_inf) || !std::isfinite(support_sup))
        return fail(RPYB_E_INVALID, "invalid support");
    if (n_events < 0) return fail(RPYB_E_INVALID, "negative event count");
    if (n_events > 0 && (!times_host || !rows)) return fail(RPYB_E_INVALID, "null event arrays");
    const int64_t lie_dim = rpyb_lie_basis_size(width, depth);
    if (lie_dim < 0) return (int)lie_dim;
    if (row_len != width && row_len != lie_dim)
        return fail(RPYB_E_INVALID, "row_len must be the width (increments) or the Lie dimension");
    for (int64_t e = 0; e < n_events; ++e) {
        if (!std::isfinite(times_host[e])) return fail(RPYB_E_INVALID, "non-finite event time");
        if (e && times_host[e] < times_host[e - 1])
            return fail(RPYB_E_INVALID, "event times must be non-decreasing");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0;
    RPYB_CUDA(cudaGetDevice(&device));

    rpyb_dyadic_tree* t = new (std::nothrow) rpyb_dyadic_tree();
    if (!t) return fail(RPYB_E_NOMEM, "out of host memory");
    t->device = device;
    t->mode = mode;
    t->width = width;
    t->depth = depth;
    t->resolution = resolution;
    t->s0 = support_inf;
    t->s1 = support_sup;
    t->g = g;
    t->lie_dim = lie_dim;

    // leaf range [m_lo, m_hi] at resolution R, covering support and events
    const int R = resolution;
    const double lo_d = std::floor(std::ldexp(support_inf, R));
    const double hi_d = std::ceil(std::ldexp(support_sup, R)) - 1.0;
    double lo_e = lo_d, hi_e = std::max(lo_d, hi_d);
    if (n_events) {
        lo_e = std::min(lo_e, std::floor(std::ldexp(times_host[0], R)));
        hi_e = std::max(hi_e, std::floor(std::ldexp(times_host[n_events - 1], R)));
    }
    if (std::fabs(lo_e) > 4.0e15 || std::fabs(hi_e) > 4.0e15 || hi_e - lo_e > 1.0e9) {
        release(t);
        return fail(RPYB_E_INVALID, "stream support too wide for its resolution");
    }
    const int64_t m_lo = (int64_t)lo_e, m_hi = (int64_t)hi_e;
    int64_t rows_total = 0;
    for (int j = 0;; ++j) {
        const int64_t l = m_lo >> j, h = m_hi >> j;
        // a range on both sides of 0 stops merging at blocks -1 and 0
        if (j > 0 && l == -1 && h == 0 && t->cnt.back() == 2) break;
        t->lo.push_back(l);
        t->cnt.push_back(h - l + 1);
        t->base.push_back(rows_total);
        rows_total += h - l + 1;
        if (h == l) break;
        if (j >= 62) {
            release(t);
            return fail(RPYB_E_INVALID, "stream support too wide for its resolution");
        }
    }
    t->J = (int)t->lo.size() - 1;
    t->unit_row = rows_total;
    t->rows = rows_total + 1;
    const int64_t T = g.size();
    const int64_t es = mode == RPYB_F64 ? 8 : 4;
    if (cudaMalloc(&t->nodes, (size_t)(t->rows * T * es)) != cudaSuccess) {
        cudaGetLastError();
        release(t);
        return fail(RPYB_E_NOMEM, "device allocation of the dyadic tree failed");
    }
    if ((rc = upload_map(width, depth, 1, lie_dim, &t->t2l_ptr, &t->t2l_idx, &t->t2l_val)) ||
        (rc = upload_map(width, depth, 0, T, &t->l2t_ptr, &t->l2t_idx, &t->l2t_val))) {
        release(t);
        return rc;
    }

    // ---- leaves
    const int64_t n_leaves = t->cnt[0];
    std::vector<int64_t> off(n_leaves + 1, 0);
    {
        int64_t e = 0;
        for (int64_t i = 0; i < n_leaves; ++i) {
            off[i] = e;
            while (e < n_events &&
                   (int64_t)std::floor(std::ldexp(times_host[e], R)) - m_lo <= i)
                ++e;
        }
        off[n_leaves] = e;
    }
    auto fail_release = [&](int code) {
        release(t);
        return code;
    };
    if (mode == RPYB_F64) {
        if ((rc = unit_rows(static_cast<double*>(t->nodes) + t->unit_row * T, T, T,
                            (const int64_t*)nullptr, 1, s)))
            return fail_release(rc);
    } else if ((rc = unit_rows(static_cast<float*>(t->nodes) + t->unit_row * T, T, T,
                               (const int64_t*)nullptr, 1, s))) {
        return fail_release(rc);
    }
    if (n_events == 0) {
        if (mode == RPYB_F64)
            rc = unit_rows(static_cast<double*>(t->nodes), T, T, (const int64_t*)nullptr, n_leaves, s);
        else
            rc = unit_rows(static_cast<float*>(t->nodes), T, T, (const int64_t*)nullptr, n_leaves, s);
        if (rc) return fail_release(rc);
    } else if (row_len == width) {
        // Chen products of exp(increment) per leaf, longest leaves first
        std::vector<int64_t> order(n_leaves);
        for (int64_t i = 0; i < n_leaves; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
            return off[a + 1] - off[a] > off[b + 1] - off[b];
        });
        const int64_t ws = rpyb_signature_workspace_size(mode, width, depth, n_leaves);
        if (ws < 0) return fail_release((int)ws);
        Scratch sc(nullptr, 0, s);
        void* mem = nullptr;
        const size_t meta = ((size_t)(2 * n_leaves + 1) * 8 + 255) / 256 * 256;
        if ((rc = sc.get(meta + (size_t)std::max<int64_t>(ws, 1), &mem))) return fail_release(rc);
        int64_t* d_off = static_cast<int64_t*>(mem);
        int64_t* d_ord = d_off + n_leaves + 1;
        std::vector<int64_t> hm(off);
        hm.insert(hm.end(), order.begin(), order.end());
        if (cudaMemcpyAsync(d_off, hm.data(), hm.size() * 8, cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
            return fail_release(cuda_fail(cudaGetLastError(), "cudaMemcpyAsync"));
        if ((rc = rpyb_signature(mode, width, depth, n_leaves, d_off, rows, t->nodes, T, d_ord,
                                 static_cast<char*>(mem) + meta, (size_t)std::max<int64_t>(ws, 1),
                                 s)))
            return fail_release(rc);
    } else {
        // Hall coordinates: exp(l2t(lie)) per event, then ordered products per leaf
        Scratch sc(nullptr, 0, s);
        void* mem = nullptr;
        const int64_t ws = rpyb_ft_exp_workspace_size(mode, width, depth, std::max<int64_t>(n_events, 1));
        const size_t emb_bytes = ((size_t)(std::max<int64_t>(n_events, 1) * T * es) + 255) / 256 * 256;
        if ((rc = sc.get(2 * emb_bytes + (size_t)std::max<int64_t>(ws, 1), &mem)))
            return fail_release(rc);
        void* emb = mem;
        void* ex = static_cast<char*>(mem) + emb_bytes;
        void* wsp = static_cast<char*>(mem) + 2 * emb_bytes;
        if (n_events) {
            if (cudaMemsetAsync(emb, 0, (size_t)(n_events * T * es), s) != cudaSuccess)
                return fail_release(cuda_fail(cudaGetLastError(), "cudaMemsetAsync"));
            if ((rc = rpyb_sparse_map(mode, T, lie_dim, n_events, t->l2t_ptr, t->l2t_idx,
                                      t->l2t_val, emb, rows, T, lie_dim, 1.0, s)) ||
                (rc = rpyb_ft_exp(mode, width, depth, n_events, ex, emb, T, T, -1, wsp,
                                  (size_t)std::max<int64_t>(ws, 1), s)))
                return fail_release(rc);
        }
        if (mode == RPYB_F64)
            rc = unit_rows(static_cast<double*>(t->nodes), T, T, (const int64_t*)nullptr, n_leaves, s);
        else
            rc = unit_rows(static_cast<float*>(t->nodes), T, T, (const int64_t*)nullptr, n_leaves, s);
        if (rc) return fail_release(rc);
        std::vector<int64_t> src(n_events);
        for (int64_t e = 0; e < n_events; ++e) src[e] = e;
        if ((rc = ordered_products(mode, mode, g, n_leaves, t->nodes, ex, off, src, s)))
            return fail_release(rc);
    }
    // ---- levels above the leaves
    if ((rc = build_levels(t, s))) return fail_release(rc);
    *out_tree = t;
    return RPYB_OK;
}

RPYB_API int rpyb_dyadic_free(rpyb_dyadic_tree* tree)
{
    release(tree);
    return RPYB_OK;
}

RPYB_API int rpyb_dyadic_tree_info(const rpyb_dyadic_tree* tree, int64_t* rows, int32_t* top_level,
                                   const void** nodes)
{
    if (!tree) return fail(RPYB_E_INVALID, "null tree");
    if (rows) *rows = tree->rows;
    if (top_level) *top_level = tree->J;
    if (nodes) *nodes = tree->nodes;
    return RPYB_OK;
}

RPYB_API int64_t rpyb_dyadic_node_row(const rpyb_dyadic_tree* tree, int32_t level, int64_t block)
{
    if (!tree) return fail(RPYB_E_INVALID, "null tree");
    return node_row(tree, level, block);
}

RPYB_API int rpyb_dyadic_query(const rpyb_dyadic_tree* t, int64_t n_queries,
                               const double* inf_host, const double* sup_host,
                               int32_t resolution, double* out_logsig, int64_t ld_logsig,
                               double* out_sig, int64_t ld_sig, void* stream)
{
    int rc;
    if (!t) return fail(RPYB_E_INVALID, "null tree");
    if (n_queries < 0) return fail(RPYB_E_INVALID, "negative query count");
    if (n_queries == 0) return RPYB_OK;
    if (!inf_host || !sup_host) return fail(RPYB_E_INVALID, "null interval arrays");
    if (!out_logsig && !out_sig) return fail(RPYB_E_INVALID, "no output requested");
    if (out_logsig && ld_logsig < t->lie_dim) return fail(RPYB_E_INVALID, "ld_logsig too small");
    if (out_sig && ld_sig < t->g.size()) return fail(RPYB_E_INVALID, "ld_sig too small");
    const bool auto_res = resolution == RPYB_QUERY_RESOLUTION_AUTO;
    if (!auto_res && (resolution < -60 || resolution > 60))
        return fail(RPYB_E_INVALID, "query resolution out of range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Geometry& g = t->g;
    const int64_t T = g.size(), L = t->lie_dim;
    const int R = t->resolution;

    // ---- host: trim to the support, choose tolerances, dissect
    // (streams/src/stream.cpp:37-71 check_support_and_trim / refine_interval)
    std::vector<double> qi(n_queries), qs(n_queries);
    std::vector<int32_t> tol(n_queries);
    std::vector<char> empty(n_queries, 0);
    int32_t max_tol = 0;
    for (int64_t q = 0; q < n_queries; ++q) {
        double a = inf_host[q], b = sup_host[q];
        if (!(a <= b)) return fail(RPYB_E_INVALID, "inf must not be larger than sup");
        if (b < t->s0 || a > t->s1) {
            empty[q] = 1;
            a = b = t->s0;
        } else {
            a = std::max(a, t->s0);
            b = std::min(b, t->s1);
        }
        if (b - a == 0.0) empty[q] = 1;
        qi[q] = a;
        qs[q] = b;
        if (auto_res)
            tol[q] = empty[q] ? R : std::max<int32_t>(R, query_param_to_resolution(b - a) + 2);
        else
            tol[q] = resolution;
        max_tol = std::max(max_tol, std::abs(tol[q]));
    }
    const int64_t cap = n_queries * (2 * (int64_t)max_tol + 130);
    std::vector<int64_t> k(cap), poff(n_queries + 1);
    std::vector<int32_t> p(cap);
    if ((rc = rpyb_dyadic_dissect_batch(n_queries, qi.data(), qs.data(), tol.data(), 1, k.data(),
                                        p.data(), cap, poff.data())))
        return rc;

    // ---- pieces -> node rows (dyadic_caching_layer.cpp:86-130): at the
    // stream resolution a leaf; coarser pieces are whole nodes; a finer piece
    // maps to the leaf it starts in when the start points coincide, and is
    // dropped otherwise.  Zero pieces are dropped.
    std::vector<int64_t> qoff(n_queries + 1, 0), nodes;
    nodes.reserve((size_t)poff[n_queries]);
    for (int64_t q = 0; q < n_queries; ++q) {
        if (!empty[q]) {
            for (int64_t i = poff[q]; i < poff[q + 1]; ++i) {
                int64_t row;
                if (p[i] <= R) {
                    row = node_row(t, (int64_t)R - p[i], k[i]);
                } else {
                    const int sh = p[i] - R;
                    if (sh > 62) {
                        row = (k[i] == 0) ? node_row(t, 0, 0) : -1;
                    } else {
                        const int64_t tk = k[i] >> sh;   // floor division
                        row = ((tk << sh) == k[i]) ? node_row(t, 0, tk) : -1;
                    }
                }
                if (row >= 0) nodes.push_back(row);
            }
        }
        qoff[q + 1] = (int64_t)nodes.size();
    }

    // ---- device, in chunks of queries bounded by a memory budget
    const int64_t budget = (int64_t)1 << 30;   // bytes per [chunk, T] float64 buffer
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(n_queries, budget / (T * 8)));
    const int64_t log_ws = rpyb_ft_log_workspace_size(RPYB_F64, g.width, g.depth, chunk);
    const int64_t exp_ws = rpyb_ft_exp_workspace_size(RPYB_F64, g.width, g.depth, chunk);
    if (log_ws < 0 || exp_ws < 0) return fail(RPYB_E_INVALID, "workspace query failed");
    const size_t buf = (size_t)((chunk * T * 8 + 255) / 256 * 256);
    const size_t lbuf = (size_t)((chunk * L * 8 + 255) / 256 * 256);
    const size_t wsb = (size_t)std::max<int64_t>(std::max(log_ws, exp_ws), 1);
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    if ((rc = sc.get(2 * buf + lbuf + wsb, &mem))) return rc;
    double* acc = static_cast<double*>(mem);
    double* tmp = reinterpret_cast<double*>(static_cast<char*>(mem) + buf);
    double* lie_tmp = reinterpret_cast<double*>(static_cast<char*>(mem) + 2 * buf);
    void* ws = static_cast<char*>(mem) + 2 * buf + lbuf;
    for (int64_t q0 = 0; q0 < n_queries; q0 += chunk) {
        const int64_t m = std::min(chunk, n_queries - q0);
        std::vector<int64_t> loff(m + 1);
        for (int64_t i = 0; i <= m; ++i) loff[i] = qoff[q0 + i] - qoff[q0];
        std::vector<int64_t> rows_q(nodes.begin() + qoff[q0], nodes.begin() + qoff[q0 + m]);
        if ((rc = unit_rows(acc, T, T, (const int64_t*)nullptr, m, s))) return rc;
        if ((rc = ordered_products(RPYB_F64, t->mode, g, m, acc, t->nodes, loff, rows_q, s)))
            return rc;
        // log in float64 (incoming out[0] must be zero), then tensor -> Lie
        RPYB_CUDA(cudaMemsetAsync(tmp, 0, (size_t)(m * T * 8), s));
        if ((rc = rpyb_ft_log(RPYB_F64, g.width, g.depth, m, tmp, acc, T, T, -1, -1, ws, wsb, s)))
            return rc;
        double* lie = out_logsig ? out_logsig + q0 * ld_logsig : lie_tmp;
        const int64_t ld_lie = out_logsig ? ld_logsig : L;
        // the sparse map accumulates: clear its outputs first
        RPYB_CUDA(cudaMemset2DAsync(lie, (size_t)(ld_lie * 8), 0, (size_t)(L * 8), (size_t)m, s));
        if ((rc = rpyb_sparse_map(RPYB_F64, L, T, m, t->t2l_ptr, t->t2l_idx, t->t2l_val, lie, tmp,
                                  ld_lie, T, 1.0, s)))
            return rc;
        if (out_sig) {
            // algebra/src/context.cpp:156-159: exp(lie_to_tensor(log_signature))
            RPYB_CUDA(cudaMemsetAsync(tmp, 0, (size_t)(m * T * 8), s));
            if ((rc = rpyb_sparse_map(RPYB_F64, T, L, m, t->l2t_ptr, t->l2t_idx, t->l2t_val, tmp,
                                      lie, T, ld_lie, 1.0, s)) ||
                (rc = rpyb_ft_exp(RPYB_F64, g.width, g.depth, m, out_sig + q0 * ld_sig, tmp,
                                  ld_sig, T, -1, ws, wsb, s)))
                return rc;
        }
    }
    return RPYB_OK;
}

}  // extern "C"
