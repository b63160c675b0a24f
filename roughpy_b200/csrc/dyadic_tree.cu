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
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "stream_ops.cuh"

struct rpyb_dyadic_tree {
    int mode = 0;
    int32_t width = 0, depth = 0, resolution = 0;
    double s0 = 0.0, s1 = 0.0;
    int device = 0;
    rpyb::Geometry g;
    int J = 0;                              // top level
    std::vector<int64_t> lo, cnt, base;     // per level: first block, blocks, first row
    int64_t unit_row = 0, rows = 0;
    void* nodes = nullptr;                  // [rows (+ table rows), T] of the mode's type
    const rpyb::LieMapsDev* maps = nullptr;
    // range-product table (rpyb_dyadic_range_table), rows after the tree's:
    // blocks of 2^tb leaves (tree level tb); pre[i] / suf[i] = product of the
    // leaves from leaf i's block start to i / from i to its block end;
    // dst[l][c] = the disjoint sparse table over the blocks (level l >= 1:
    // the product from block c to the middle of its 2^l group, or from the
    // middle to c)
    int tb = -1;
    int64_t pre_base = 0, suf_base = 0, dst_base = 0;
    int dst_levels = 0;
};

namespace rpyb {
namespace {

// Saved form of a tree (rpyb_dyadic_save / rpyb_dyadic_load): this header,
// then the per-level tables lo[J+1], cnt[J+1], base[J+1] (int64), then the
// node table [rows, tensor_size] of the mode's type, all in host byte order.
constexpr char kTreeMagic[8] = {'R', 'P', 'Y', 'B', 'D', 'Y', 'T', '1'};
constexpr int64_t kTreeVersion = 1;
struct SavedTreeHeader {
    char magic[8];
    int64_t version;
    int64_t mode, width, depth, resolution;
    double support_inf, support_sup;
    int64_t top_level, unit_row, rows, tensor_size, elem_bytes;
    int64_t reserved[4];
};

void release(rpyb_dyadic_tree* t)
{
    if (!t) return;
    if (t->nodes) {
        int cur = 0;
        const bool switched = cudaGetDevice(&cur) == cudaSuccess && cur != t->device &&
                              cudaSetDevice(t->device) == cudaSuccess;
        cudaFree(t->nodes);
        if (switched) cudaSetDevice(cur);
    }
    delete t;
}

int64_t node_row(const rpyb_dyadic_tree* t, int64_t level, int64_t blk)
{
    if (level < 0 || level > t->J) return -1;
    const int64_t rel = blk - t->lo[level];
    if (rel < 0 || rel >= t->cnt[level]) return -1;
    return t->base[level] + rel;
}

// Tree rows covering the leaf range [a, e) in order (greedy maximal aligned
// blocks; blocks the tree does not hold, outside the leaf range, are units
// and skipped).
void range_nodes(const rpyb_dyadic_tree* t, int64_t a, int64_t e, std::vector<int64_t>& out)
{
    const int64_t l0 = t->lo[0], h0 = t->lo[0] + t->cnt[0];
    while (a < e) {
        int j;
        if (a >= l0 && a < h0) {
            // the tree holds every block containing a leaf of its range: the
            // block is the largest one aligned at a that fits [a, e)
            const int tz = a == 0 ? 62 : __builtin_ctzll((unsigned long long)a);
            const int lg = 63 - __builtin_clzll((unsigned long long)(e - a));
            j = std::min(std::min(tz, lg), (int)t->J);
        } else {
            j = 0;
            while (j < t->J && (a >> (j + 1)) * ((int64_t)2 << j) == a &&
                   a + ((int64_t)2 << j) <= e && node_row(t, j + 1, a >> (j + 1)) >= 0)
                ++j;
        }
        const int64_t row = node_row(t, j, a >> j);
        if (row >= 0) out.push_back(row);
        a += (int64_t)1 << j;
    }
}

// Leaves of at most one level-1 event: exp(x) written directly, one warp per
// leaf.  Word (a_1 .. a_k) of exp(x) is x_{a_1} ... x_{a_k} / k!; the words of
// level depth-1 are formed once and extended by every last letter for the
// top level.  Computed in float64, rounded once to the tree's type; an empty
// leaf is the unit.
struct LeafExpArgs {
    int32_t width = 0, depth = 0;
    int64_t T = 0;
    int64_t db[kMaxDepth + 2] = {};
    int64_t pw[kMaxDepth + 1] = {};
    double inv_fact[kMaxDepth + 1] = {};
};

template <typename T>
__global__ void leaf_exp_kernel(const LeafExpArgs a, T* __restrict__ nodes,
                                const T* __restrict__ rows, const int64_t* __restrict__ off,
                                int64_t n_leaves)
{
    __shared__ double xs_all[8][16];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double* xs = xs_all[wib];
    const int d = a.width, N = a.depth;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t leaf = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib; leaf < n_leaves;
         leaf += nwarps) {
        T* __restrict__ o = nodes + leaf * a.T;
        const int64_t e0 = off[leaf];
        __syncwarp();
        if (off[leaf + 1] == e0) {
            for (int64_t i = lane; i < a.T; i += 32) o[i] = (i == 0) ? T(1) : T(0);
            continue;
        }
        if (lane < d) xs[lane] = (double)rows[e0 * d + lane];
        __syncwarp();
        // levels 0 .. depth-1 word by word
        for (int k = 0; k <= N - 1; ++k) {
            const int64_t nk = a.pw[k];
            for (int64_t w = lane; w < nk; w += 32) {
                double v = a.inv_fact[k];
                int64_t r = w;
                for (int i = 0; i < k; ++i) {
                    const int64_t q = r / d;
                    v *= xs[r - q * d];
                    r = q;
                }
                o[a.db[k] + w] = (T)v;
                if (k == N - 1 && N >= 1) {
                    // the top level: (w, b) = word w * x_b / N
                    const double p = v / (double)N;
                    T* top = o + a.db[N] + w * d;
                    for (int b = 0; b < d; ++b) top[b] = (T)(p * xs[b]);
                }
            }
        }
    }
}

// float64 accumulator rows acc[i] -> tree-typed rows dst[i] (mode's type)
template <typename T>
__global__ void store_rows_kernel(T* __restrict__ nodes, int64_t T_, const double* __restrict__ acc,
                                  const int64_t* __restrict__ dst, int64_t n)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * T_;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / T_, c = e - r * T_;
        nodes[dst[r] * T_ + c] = (T)acc[e];
    }
}

// the most events any leaf holds
int64_t max_leaf_events(const std::vector<int64_t>& off)
{
    int64_t most = 0;
    for (size_t i = 0; i + 1 < off.size(); ++i) most = std::max(most, off[i + 1] - off[i]);
    return most;
}

int build_levels(rpyb_dyadic_tree* t, cudaStream_t s)
{
    const Geometry& g = t->g;
    std::vector<int64_t> packed, start(t->J + 2, 0);
    for (int j = 1; j <= t->J; ++j) {
        start[j] = (int64_t)packed.size();
        const int64_t n = t->cnt[j];
        auto row = [&](int64_t c) {
            const int64_t rel = c - t->lo[j - 1];
            return (rel >= 0 && rel < t->cnt[j - 1]) ? t->base[j - 1] + rel : t->unit_row;
        };
        for (int64_t i = 0; i < n; ++i) packed.push_back(t->base[j] + i);
        for (int64_t i = 0; i < n; ++i) packed.push_back(row(2 * (t->lo[j] + i)));
        for (int64_t i = 0; i < n; ++i) packed.push_back(row(2 * (t->lo[j] + i) + 1));
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
    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;

    // leaf range [m_lo, m_hi] at resolution R, covering support and events
    const int R = resolution;
    const double lo_d = std::floor(std::ldexp(support_inf, R));
    const double hi_d = std::ceil(std::ldexp(support_sup, R)) - 1.0;
    double lo_e = lo_d, hi_e = std::max(lo_d, hi_d);
    if (n_events) {
        lo_e = std::min(lo_e, std::floor(std::ldexp(times_host[0], R)));
        hi_e = std::max(hi_e, std::floor(std::ldexp(times_host[n_events - 1], R)));
    }
    if (std::fabs(lo_e) > 4.0e15 || std::fabs(hi_e) > 4.0e15 || hi_e - lo_e > 1.0e9)
        return fail(RPYB_E_INVALID, "stream support too wide for its resolution");

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
    t->maps = maps;
    auto fail_release = [&](int code) {
        release(t);
        return code;
    };

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
        if (j >= 62)
            return fail_release(fail(RPYB_E_INVALID, "stream support too wide for its resolution"));
    }
    t->J = (int)t->lo.size() - 1;
    t->unit_row = rows_total;
    t->rows = rows_total + 1;
    const int64_t T = g.size();
    const int64_t es = mode == RPYB_F64 ? 8 : 4;
    if (cudaMalloc(&t->nodes, (size_t)(t->rows * T * es)) != cudaSuccess) {
        cudaGetLastError();
        t->nodes = nullptr;
        return fail_release(fail(RPYB_E_NOMEM, "device allocation of the dyadic tree failed"));
    }

    // ---- leaves: events grouped by leaf (times are sorted)
    const int64_t n_leaves = t->cnt[0];
    std::vector<int64_t> off(n_leaves + 1, 0);
    {
        int64_t e = 0;
        for (int64_t i = 0; i < n_leaves; ++i) {
            off[i] = e;
            while (e < n_events && (int64_t)std::floor(std::ldexp(times_host[e], R)) - m_lo <= i)
                ++e;
        }
        off[n_leaves] = e;
    }
    if ((rc = unit_rows(mode, static_cast<char*>(t->nodes) + t->unit_row * T * es, T, T, nullptr,
                        1, s)))
        return fail_release(rc);
    if (n_events == 0) {
        if ((rc = unit_rows(mode, t->nodes, T, T, nullptr, n_leaves, s))) return fail_release(rc);
    } else if (row_len == width && max_leaf_events(off) <= 1 && width <= 16) {
        // at most one event per leaf: exp(x) directly
        LeafExpArgs la;
        la.width = width;
        la.depth = depth;
        la.T = T;
        for (int k = 0; k <= kMaxDepth + 1; ++k) la.db[k] = g.db[k];
        double f = 1.0;
        for (int k = 0; k <= kMaxDepth; ++k) {
            la.pw[k] = g.pw[k];
            if (k > 0) f *= (double)k;
            la.inv_fact[k] = 1.0 / f;
        }
        Scratch sc(nullptr, 0, s);
        void* mem = nullptr;
        if ((rc = sc.get((size_t)(n_leaves + 1) * 8, &mem))) return fail_release(rc);
        int64_t* d_off = static_cast<int64_t*>(mem);
        if (cudaMemcpyAsync(d_off, off.data(), (size_t)(n_leaves + 1) * 8, cudaMemcpyHostToDevice,
                            s) != cudaSuccess)
            return fail_release(cuda_fail(cudaGetLastError(), "cudaMemcpyAsync"));
        const unsigned blocks = (unsigned)std::min<int64_t>((n_leaves + 7) / 8, 148 * 64);
        if (mode == RPYB_F64)
            leaf_exp_kernel<double><<<blocks, 256, 0, s>>>(
                la, static_cast<double*>(t->nodes), static_cast<const double*>(rows), d_off,
                n_leaves);
        else
            leaf_exp_kernel<float><<<blocks, 256, 0, s>>>(
                la, static_cast<float*>(t->nodes), static_cast<const float*>(rows), d_off,
                n_leaves);
        if (cudaGetLastError() != cudaSuccess)
            return fail_release(fail(RPYB_E_CUDA, "leaf_exp_kernel launch"));
        // the host offsets must outlive the asynchronous copy
        if (cudaStreamSynchronize(s) != cudaSuccess)
            return fail_release(cuda_fail(cudaGetLastError(), "cudaStreamSynchronize"));
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
        const int64_t ws = rpyb_ft_exp_workspace_size(mode, width, depth, n_events);
        const size_t emb_bytes = ((size_t)(n_events * T * es) + 255) / 256 * 256;
        if ((rc = sc.get(2 * emb_bytes + (size_t)std::max<int64_t>(ws, 1), &mem)))
            return fail_release(rc);
        void* emb = mem;
        void* ex = static_cast<char*>(mem) + emb_bytes;
        void* wsp = static_cast<char*>(mem) + 2 * emb_bytes;
        // the sparse map accumulates: clear its output first
        if (cudaMemsetAsync(emb, 0, (size_t)(n_events * T * es), s) != cudaSuccess)
            return fail_release(cuda_fail(cudaGetLastError(), "cudaMemsetAsync"));
        if ((rc = rpyb_sparse_map(mode, T, lie_dim, n_events, maps->l2t_ptr, maps->l2t_idx,
                                  maps->l2t_val, emb, rows, T, lie_dim, 1.0, s)) ||
            (rc = rpyb_ft_exp(mode, width, depth, n_events, ex, emb, T, T, -1, wsp,
                              (size_t)std::max<int64_t>(ws, 1), s)) ||
            (rc = unit_rows(mode, t->nodes, T, T, nullptr, n_leaves, s)))
            return fail_release(rc);
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

RPYB_API int rpyb_dyadic_range_table(rpyb_dyadic_tree* t, int32_t block_log2, void* stream)
{
    int rc;
    if (!t) return fail(RPYB_E_INVALID, "null tree");
    if (block_log2 < 0 || block_log2 > 30) return fail(RPYB_E_INVALID, "block_log2 out of range");
    const int64_t n0 = t->cnt[0];
    int b = block_log2;
    if (b == 0) {
        // blocks of about sqrt(leaves), at least 16 leaves
        b = 4;
        while (b < 30 && ((int64_t)1 << (2 * (b + 1))) <= n0) ++b;
    }
    if (t->tb >= 0) return RPYB_OK;                       // already built
    if (b > t->J || n0 < ((int64_t)4 << b)) return RPYB_OK;  // too small to pay off
    const Geometry& g = t->g;
    const int64_t T = g.size();
    const int64_t es = t->mode == RPYB_F64 ? 8 : 4;
    const int64_t nb = t->cnt[b], lob = t->lo[b], lo0 = t->lo[0];
    int levels = 0;
    while (((int64_t)1 << levels) < nb) ++levels;
    // factor lists (tree rows) of every table entry, in table-row order
    std::vector<int64_t> off{0}, rows_list;
    off.reserve(2 * n0 + (size_t)levels * nb + 1);
    for (int side = 0; side < 2; ++side) {
        for (int64_t i = 0; i < n0; ++i) {
            const int64_t k = lo0 + i;
            const int64_t bs = std::max((k >> b) * ((int64_t)1 << b), lo0);
            const int64_t be = std::min(((k >> b) + 1) * ((int64_t)1 << b), lo0 + n0);
            if (side == 0) range_nodes(t, bs, k + 1, rows_list);   // pre
            else range_nodes(t, k, be, rows_list);                 // suf
            off.push_back((int64_t)rows_list.size());
        }
    }
    for (int l = 1; l <= levels; ++l) {
        for (int64_t c = 0; c < nb; ++c) {
            const int64_t half = (int64_t)1 << (l - 1);
            const int64_t mid = ((c >> l) << l) + half;
            // blocks [c, mid) on the left of the middle, [mid, c] on the right
            const int64_t c0 = c < mid ? c : mid, c1 = c < mid ? std::min(mid, nb) : c + 1;
            const int64_t B = (int64_t)1 << b;
            range_nodes(t, std::max((lob + c0) * B, lo0), std::min((lob + c1) * B, lo0 + n0),
                        rows_list);
            off.push_back((int64_t)rows_list.size());
        }
    }
    const int64_t extra = (int64_t)off.size() - 1;
    // a new node table with room for the table rows; the tree rows move over
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void* grown = nullptr;
    if (cudaMalloc(&grown, (size_t)((t->rows + extra) * T * es)) != cudaSuccess) {
        cudaGetLastError();
        return fail(RPYB_E_NOMEM, "device allocation of the range table failed");
    }
    if (cudaMemcpyAsync(grown, t->nodes, (size_t)(t->rows * T * es), cudaMemcpyDeviceToDevice,
                        s) != cudaSuccess) {
        rc = cuda_fail(cudaGetLastError(), "cudaMemcpyAsync");
        cudaFree(grown);
        return rc;
    }
    void* old_nodes = t->nodes;
    // products in chunks, accumulated in float64 on the device and rounded
    // once to the tree's type
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(8192, ((int64_t)1 << 30) / (T * 8)));
    const bool chain = chain_products_available(g);
    std::vector<int64_t> loff, lrows, dst;
    if (chain) {
        // the chain kernel writes the table rows straight into the grown
        // node table; its index lists are copied when the call returns, so
        // the host prepares the next chunk while the device runs this one
        for (int64_t e0 = 0; e0 < extra && rc == RPYB_OK; e0 += chunk) {
            const int64_t m = std::min(chunk, extra - e0);
            loff.assign(m + 1, 0);
            for (int64_t i = 0; i <= m; ++i) loff[i] = off[e0 + i] - off[e0];
            lrows.assign(rows_list.begin() + off[e0], rows_list.begin() + off[e0 + m]);
            dst.resize(m);
            for (int64_t i = 0; i < m; ++i) dst[i] = t->rows + e0 + i;
            rc = chain_products_into(t->mode, g, m, grown, loff, lrows, dst, s);
        }
    } else {
        Scratch sc(nullptr, 0, s);
        void* mem = nullptr;
        if ((rc = sc.get((size_t)(chunk * T * 8 + chunk * 8 + 256), &mem))) {
            cudaFree(grown);
            return rc;
        }
        double* acc = static_cast<double*>(mem);
        int64_t* d_dst = reinterpret_cast<int64_t*>(static_cast<char*>(mem) + chunk * T * 8);
        for (int64_t e0 = 0; e0 < extra && rc == RPYB_OK; e0 += chunk) {
            const int64_t m = std::min(chunk, extra - e0);
            loff.assign(m + 1, 0);
            for (int64_t i = 0; i <= m; ++i) loff[i] = off[e0 + i] - off[e0];
            lrows.assign(rows_list.begin() + off[e0], rows_list.begin() + off[e0 + m]);
            dst.resize(m);
            for (int64_t i = 0; i < m; ++i) dst[i] = t->rows + e0 + i;
            rc = unit_rows(RPYB_F64, acc, T, T, nullptr, m, s);
            if (!rc) rc = ordered_products(RPYB_F64, t->mode, g, m, acc, grown, loff, lrows, s);
            if (rc) break;
            if (cudaMemcpyAsync(d_dst, dst.data(), (size_t)m * 8, cudaMemcpyHostToDevice, s) !=
                cudaSuccess) {
                rc = cuda_fail(cudaGetLastError(), "cudaMemcpyAsync");
                break;
            }
            const unsigned blocks = (unsigned)std::min<int64_t>((m * T + 255) / 256, 148 * 32);
            if (t->mode == RPYB_F64)
                store_rows_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double*>(grown), T,
                                                                 acc, d_dst, m);
            else
                store_rows_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float*>(grown), T,
                                                                acc, d_dst, m);
            if (cudaGetLastError() != cudaSuccess) rc = fail(RPYB_E_CUDA, "store_rows_kernel launch");
            // the host vectors are reused by the next chunk: wait for the copy
            if (!rc && cudaStreamSynchronize(s) != cudaSuccess)
                rc = cuda_fail(cudaGetLastError(), "cudaStreamSynchronize");
        }
    }
    if (rc) {
        cudaStreamSynchronize(s);
        cudaFree(grown);
        return rc;
    }
    RPYB_CUDA(cudaStreamSynchronize(s));
    cudaFree(old_nodes);
    t->nodes = grown;
    t->tb = b;
    t->pre_base = t->rows;
    t->suf_base = t->rows + n0;
    t->dst_base = t->rows + 2 * n0;
    t->dst_levels = levels;
    return RPYB_OK;
}

RPYB_API int64_t rpyb_dyadic_save_size(const rpyb_dyadic_tree* t)
{
    if (!t) return fail(RPYB_E_INVALID, "null tree");
    const int64_t es = t->mode == RPYB_F64 ? 8 : 4;
    return (int64_t)sizeof(SavedTreeHeader) + 3 * (int64_t)(t->J + 1) * 8 +
           t->rows * t->g.size() * es;
}

RPYB_API int64_t rpyb_dyadic_save(const rpyb_dyadic_tree* t, void* buf, int64_t cap, void* stream)
{
    if (!t) return fail(RPYB_E_INVALID, "null tree");
    const int64_t need = rpyb_dyadic_save_size(t);
    if (!buf || cap < need)
        return fail(RPYB_E_INVALID, "save buffer too small: need " + std::to_string(need) + " bytes");
    SavedTreeHeader h{};
    memcpy(h.magic, kTreeMagic, sizeof h.magic);
    h.version = kTreeVersion;
    h.mode = t->mode;
    h.width = t->width;
    h.depth = t->depth;
    h.resolution = t->resolution;
    h.support_inf = t->s0;
    h.support_sup = t->s1;
    h.top_level = t->J;
    h.unit_row = t->unit_row;
    h.rows = t->rows;
    h.tensor_size = t->g.size();
    h.elem_bytes = t->mode == RPYB_F64 ? 8 : 4;
    char* out = static_cast<char*>(buf);
    memcpy(out, &h, sizeof h);
    int64_t* arr = reinterpret_cast<int64_t*>(out + sizeof h);
    for (int j = 0; j <= t->J; ++j) {
        arr[j] = t->lo[j];
        arr[t->J + 1 + j] = t->cnt[j];
        arr[2 * (t->J + 1) + j] = t->base[j];
    }
    char* nodes = out + sizeof h + 3 * (int64_t)(t->J + 1) * 8;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RPYB_CUDA(cudaMemcpyAsync(nodes, t->nodes, (size_t)(t->rows * h.tensor_size * h.elem_bytes),
                              cudaMemcpyDeviceToHost, s));
    RPYB_CUDA(cudaStreamSynchronize(s));
    return need;
}

RPYB_API int rpyb_dyadic_load(const void* buf, int64_t size, rpyb_dyadic_tree** out_tree,
                              void* stream)
{
    int rc;
    if (!out_tree) return fail(RPYB_E_INVALID, "null tree handle");
    *out_tree = nullptr;
    if (!buf || size < (int64_t)sizeof(SavedTreeHeader))
        return fail(RPYB_E_INVALID, "not a saved dyadic tree (too short)");
    SavedTreeHeader h;
    memcpy(&h, buf, sizeof h);
    if (memcmp(h.magic, kTreeMagic, sizeof h.magic) != 0)
        return fail(RPYB_E_INVALID, "not a saved dyadic tree (bad magic)");
    if (h.version != kTreeVersion) return fail(RPYB_E_INVALID, "unsupported saved-tree version");
    if (h.mode != RPYB_F32 && h.mode != RPYB_F64) return fail(RPYB_E_INVALID, "bad saved mode");
    Geometry g;
    if (h.width < 1 || h.width > (1 << 20) || h.depth < 0 || h.depth > kMaxDepth ||
        make_geometry((int32_t)h.width, (int32_t)h.depth, g))
        return fail(RPYB_E_INVALID, "bad saved tensor shape");
    if (h.tensor_size != g.size() || h.elem_bytes != (h.mode == RPYB_F64 ? 8 : 4) ||
        h.top_level < 0 || h.top_level > 62 || h.rows < 1 || h.unit_row != h.rows - 1)
        return fail(RPYB_E_INVALID, "inconsistent saved-tree header");
    const int64_t J = h.top_level;
    const int64_t need = (int64_t)sizeof h + 3 * (J + 1) * 8 + h.rows * h.tensor_size * h.elem_bytes;
    if (size != need) return fail(RPYB_E_INVALID, "saved-tree size does not match its header");
    const int64_t* arr = reinterpret_cast<const int64_t*>(static_cast<const char*>(buf) + sizeof h);
    int64_t acc = 0;
    for (int64_t j = 0; j <= J; ++j) {
        if (arr[J + 1 + j] < 1 || arr[2 * (J + 1) + j] != acc)
            return fail(RPYB_E_INVALID, "inconsistent saved-tree level table");
        acc += arr[J + 1 + j];
    }
    if (acc != h.unit_row) return fail(RPYB_E_INVALID, "inconsistent saved-tree level table");
    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;
    rpyb_dyadic_tree* t = new (std::nothrow) rpyb_dyadic_tree();
    if (!t) return fail(RPYB_E_NOMEM, "out of host memory");
    if (cudaGetDevice(&t->device) != cudaSuccess) {
        delete t;
        return cuda_fail(cudaGetLastError(), "cudaGetDevice");
    }
    t->mode = (int)h.mode;
    t->width = (int32_t)h.width;
    t->depth = (int32_t)h.depth;
    t->resolution = (int32_t)h.resolution;
    t->s0 = h.support_inf;
    t->s1 = h.support_sup;
    t->g = g;
    t->maps = maps;
    t->J = (int)J;
    t->unit_row = h.unit_row;
    t->rows = h.rows;
    for (int64_t j = 0; j <= J; ++j) {
        t->lo.push_back(arr[j]);
        t->cnt.push_back(arr[J + 1 + j]);
        t->base.push_back(arr[2 * (J + 1) + j]);
    }
    const size_t bytes = (size_t)(h.rows * h.tensor_size * h.elem_bytes);
    if (cudaMalloc(&t->nodes, bytes) != cudaSuccess) {
        cudaGetLastError();
        t->nodes = nullptr;
        release(t);
        return fail(RPYB_E_NOMEM, "device allocation of the dyadic tree failed");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const char* nodes = static_cast<const char*>(buf) + sizeof h + 3 * (J + 1) * 8;
    if (cudaMemcpyAsync(t->nodes, nodes, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        rc = cuda_fail(cudaGetLastError(), "cudaMemcpyAsync");
        release(t);
        return rc;
    }
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
    const Geometry& g = t->g;
    const int64_t T = g.size(), L = t->maps->lie_dim;
    if (out_logsig && ld_logsig < L) return fail(RPYB_E_INVALID, "ld_logsig too small");
    if (out_sig && ld_sig < T) return fail(RPYB_E_INVALID, "ld_sig too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int R = t->resolution;

    // device buffers for chunks of queries bounded by a memory budget; the
    // host work of a chunk (trim, dissection, node lookup) overlaps the
    // device work of the previous one
    const int64_t budget = (int64_t)1 << 30;   // bytes per [chunk, T] float64 buffer
    const int64_t chunk = std::max<int64_t>(
        1, std::min<int64_t>({n_queries, budget / (T * 8), (int64_t)8192}));
    const size_t buf = (size_t)((chunk * T * 8 + 255) / 256 * 256);
    const size_t fin = finish_scratch_bytes(g, L, chunk);
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    if ((rc = sc.get(buf + fin, &mem))) return rc;
    double* acc = static_cast<double*>(mem);
    void* fin_mem = static_cast<char*>(mem) + buf;
    std::vector<int64_t> k, poff, qoff, nodes;
    std::vector<int32_t> p;
    for (int64_t q0 = 0; q0 < n_queries; q0 += chunk) {
        const int64_t m = std::min(chunk, n_queries - q0);
        if ((rc = refine_and_dissect(m, inf_host + q0, sup_host + q0, t->s0, t->s1, R, resolution,
                                     k, p, poff)))
            return rc;
        // pieces -> node rows (dyadic_caching_layer.cpp:86-130): at the
        // stream resolution a leaf; coarser pieces are whole nodes; a finer
        // piece maps to the leaf it starts in when the start points
        // coincide, and is dropped otherwise.  Zero pieces are dropped.
        qoff.assign(m + 1, 0);
        nodes.clear();
        for (int64_t q = 0; q < m; ++q) {
            if (t->tb >= 0 && poff[q + 1] > poff[q]) {
                // with the range table: pieces no finer than the leaves cover the
                // leaf range [la, lb); across blocks it is at most four factors
                bool coarse = true;
                for (int64_t i = poff[q]; i < poff[q + 1]; ++i)
                    coarse = coarse && p[i] <= R && R - p[i] <= 40;
                if (coarse) {
                    const int64_t i0 = poff[q], i1 = poff[q + 1] - 1;
                    const int64_t lo0 = t->lo[0], hi0 = t->lo[0] + t->cnt[0];
                    const int64_t la = std::max(k[i0] * ((int64_t)1 << (R - p[i0])), lo0);
                    const int64_t lb = std::min((k[i1] + 1) * ((int64_t)1 << (R - p[i1])), hi0);
                    const int b = t->tb;
                    if (la < lb && (la >> b) != ((lb - 1) >> b)) {
                        const int64_t A = la >> b, Bk = (lb - 1) >> b;
                        const bool la_al = (la >> b) * ((int64_t)1 << b) == la;
                        const bool lb_al = (lb >> b) * ((int64_t)1 << b) == lb;
                        if (!la_al) nodes.push_back(t->suf_base + (la - lo0));
                        const int64_t A1 = A + (la_al ? 0 : 1), B1 = Bk - (lb_al ? 0 : 1);
                        if (A1 == B1) {
                            nodes.push_back(node_row(t, b, A1));
                        } else if (A1 < B1) {
                            const int64_t ra = A1 - t->lo[b], rb = B1 - t->lo[b];
                            const int l = 64 - __builtin_clzll((unsigned long long)(ra ^ rb));
                            const int64_t nb = t->cnt[b];
                            nodes.push_back(t->dst_base + (int64_t)(l - 1) * nb + ra);
                            nodes.push_back(t->dst_base + (int64_t)(l - 1) * nb + rb);
                        }
                        if (!lb_al) nodes.push_back(t->pre_base + (lb - 1 - lo0));
                        qoff[q + 1] = (int64_t)nodes.size();
                        continue;
                    }
                }
            }
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
            qoff[q + 1] = (int64_t)nodes.size();
        }
        const bool chain = chain_products_available(g);
        double* lsq = out_logsig ? out_logsig + q0 * ld_logsig : nullptr;
        if (chain && chain_lie_available(g, *t->maps)) {
            // chain products, log and Hall projection in one kernel
            int64_t ld_lie = 0;
            double* lie = finish_lie_rows(g, t->maps->lie_dim, m, fin_mem, lsq, ld_logsig, &ld_lie);
            if ((rc = chain_products_lie(t->mode, g, m, t->nodes, qoff, nodes, *t->maps, lie,
                                         ld_lie, s)) ||
                (rc = finish_queries(g, *t->maps, m, acc, true, lsq, ld_logsig,
                                     out_sig ? out_sig + q0 * ld_sig : nullptr, ld_sig, fin_mem,
                                     fin, s, true)))
                return rc;
            continue;
        }
        if ((rc = chain ? chain_products(t->mode, g, m, acc, t->nodes, qoff, nodes, true, s)
                        : (unit_rows(RPYB_F64, acc, T, T, nullptr, m, s) ||
                           ordered_products(RPYB_F64, t->mode, g, m, acc, t->nodes, qoff, nodes,
                                            s))) ||
            (rc = finish_queries(g, *t->maps, m, acc, chain, lsq, ld_logsig,
                                 out_sig ? out_sig + q0 * ld_sig : nullptr, ld_sig, fin_mem, fin,
                                 s)))
            return rc;
    }
    return RPYB_OK;
}

}  // extern "C"
