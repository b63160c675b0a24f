// Shared stream building blocks (see stream_ops.cuh).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "stream_ops.cuh"

namespace rpyb {
namespace {

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

// acc[order[i]] <- (parity[i] ? b1 : b0)[i] for i < n (rows of `cols` values)
template <typename T>
__global__ void gather_final_kernel(T* __restrict__ acc, const T* __restrict__ b0,
                                    const T* __restrict__ b1, int64_t cols,
                                    const int64_t* __restrict__ order,
                                    const int64_t* __restrict__ parity, int64_t n)
{
    const int64_t total = n * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / cols, c = e - i * cols;
        const T* src = parity[i] ? b1 : b0;
        acc[order[i] * cols + c] = src[i * cols + c];
    }
}

unsigned grid_for(int64_t total)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
}

// streams/include/roughpy/streams/stream_base.h:74-83 (query_resolution)
int32_t query_param_to_resolution(double length)
{
    int e = 0;
    std::frexp(length, &e);
    return -std::min(0, e - 1);
}

int upload_csr(const Geometry& g, int which, int64_t n_rows, const int64_t** ptr,
               const int64_t** idx, const double** val)
{
    const int64_t nnz = rpyb_lie_map_csr(g.width, g.depth, which, nullptr, nullptr, nullptr);
    if (nnz < 0) return (int)nnz;
    std::vector<int64_t> hp(n_rows + 1), hi(std::max<int64_t>(nnz, 1));
    std::vector<double> hv(std::max<int64_t>(nnz, 1));
    const int64_t got = rpyb_lie_map_csr(g.width, g.depth, which, hp.data(), hi.data(), hv.data());
    if (got < 0) return (int)got;
    int64_t* dp = nullptr;
    int64_t* di = nullptr;
    double* dv = nullptr;
    RPYB_CUDA(cudaMalloc(&dp, hp.size() * 8));
    RPYB_CUDA(cudaMalloc(&di, hi.size() * 8));
    RPYB_CUDA(cudaMalloc(&dv, hv.size() * 8));
    RPYB_CUDA(cudaMemcpy(dp, hp.data(), hp.size() * 8, cudaMemcpyHostToDevice));
    RPYB_CUDA(cudaMemcpy(di, hi.data(), hi.size() * 8, cudaMemcpyHostToDevice));
    RPYB_CUDA(cudaMemcpy(dv, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice));
    *ptr = dp;
    *idx = di;
    *val = dv;
    return RPYB_OK;
}

// Pinned staging for host -> device uploads of index lists.  A copy from
// pageable memory makes cudaMemcpyAsync wait for the stream, which would
// serialise the host work of the next query chunk behind the device work of
// the previous one.  Two pinned buffers per host thread and device
// alternate; an event per buffer marks when its last copy has completed.
struct PinnedStage {
    void* p = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
};

int upload_async(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    thread_local PinnedStage stages[64][2];
    thread_local int next[64] = {};
    int dev = 0;
    RPYB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(RPYB_E_UNSUPPORTED, "device ordinal too large");
    PinnedStage& st = stages[dev][next[dev]];
    next[dev] ^= 1;
    if (st.ev) RPYB_CUDA(cudaEventSynchronize(st.ev));   // its previous copy is done
    if (st.cap < bytes) {
        if (st.p) RPYB_CUDA(cudaFreeHost(st.p));
        st.p = nullptr;
        st.cap = 0;
        const size_t cap = std::max<size_t>(bytes + bytes / 2, 1 << 20);
        RPYB_CUDA(cudaMallocHost(&st.p, cap));
        st.cap = cap;
    }
    if (!st.ev) RPYB_CUDA(cudaEventCreateWithFlags(&st.ev, cudaEventDisableTiming));
    std::memcpy(st.p, src, bytes);
    RPYB_CUDA(cudaMemcpyAsync(dst, st.p, bytes, cudaMemcpyHostToDevice, s));
    RPYB_CUDA(cudaEventRecord(st.ev, s));
    return RPYB_OK;
}


// ------------------------------------------------------------------------
// Fused chain products: one block per row q keeps acc[q] in shared memory
// (float64, double-buffered) and multiplies in the rows src[r] of its list
// one after the other, so the accumulator crosses HBM once instead of once
// per factor.  A product is split like the blocked product kernel: a unit
// owns D first letters x V last letters of one middle part at a level
// k >= 2; levels 0 and 1 are done by the first threads.
struct ChainArgs {
    int64_t T = 0;
    int64_t db[kMaxDepth + 2] = {};
    int64_t pw[kMaxDepth + 1] = {};
    int64_t ucum[kMaxDepth + 2] = {};   // work units before level k (k >= 2)
    int64_t utotal = 0;
    int depth = 0;
    int64_t n = 0;
    const int64_t* off = nullptr;      // [n + 1] into rows
    const int64_t* rows = nullptr;     // source row of each factor
    const void* src = nullptr;         // [*, T] factors (float or double)
    double* acc = nullptr;             // [n, T] in/out
};

constexpr int kChainThreads = 512;

template <typename TS, int D, int V>
__global__ void __launch_bounds__(kChainThreads, 1)
chain_products_kernel(const ChainArgs a)
{
    constexpr int NB = D / V;
    extern __shared__ __align__(16) unsigned char chain_smem[];
    double* buf0 = reinterpret_cast<double*>(chain_smem);
    double* buf1 = buf0 + a.T;
    const int tid = (int)threadIdx.x;
    const TS* src = static_cast<const TS*>(a.src);
    for (int64_t q = blockIdx.x; q < a.n; q += gridDim.x) {
        const int64_t o0 = a.off[q], o1 = a.off[q + 1];
        if (o0 == o1) continue;
        double* accq = a.acc + q * a.T;
        double* cur = buf0;
        double* nxt = buf1;
        __syncthreads();
        for (int64_t i = tid; i < a.T; i += blockDim.x) cur[i] = accq[i];
        __syncthreads();
        for (int64_t r = o0; r < o1; ++r) {
            const TS* node = src + a.rows[r] * a.T;
            const double node0 = (double)__ldg(node);
            const double c0v = cur[0];
            if (tid == 0) nxt[0] = c0v * node0;
            if (tid < D) nxt[1 + tid] = cur[1 + tid] * node0 + c0v * (double)__ldg(node + 1 + tid);
            for (int64_t f = tid; f < a.utotal; f += blockDim.x) {
                int k = 2;
                while (f >= a.ucum[k + 1]) ++k;
                const int64_t unit = f - a.ucum[k];
                const uint32_t rp = (uint32_t)(unit / NB);
                const int c0 = (int)(unit - (int64_t)rp * NB) * V;
                const int64_t dk1 = a.pw[k - 1];
                const int64_t obase = a.db[k] + (int64_t)rp * D + c0;
                double acc[D][V];
#pragma unroll
                for (int u = 0; u < D; ++u)
#pragma unroll
                    for (int j = 0; j < V; ++j) acc[u][j] = cur[obase + u * dk1 + j] * node0;
                uint32_t qq = rp;
                uint32_t m = 0;
                for (int s = 1; s <= k - 1; ++s) {
                    const int p = k - s;
                    double lv[D];
                    double rv[V];
                    const double* lp = cur + a.db[p] + qq;
                    const uint32_t dp1 = (uint32_t)a.pw[p - 1];
#pragma unroll
                    for (int u = 0; u < D; ++u) lv[u] = lp[u * dp1];
                    const TS* rq = node + a.db[s] + (int64_t)m * D + c0;
#pragma unroll
                    for (int j = 0; j < V; ++j) rv[j] = (double)__ldg(rq + j);
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j) acc[u][j] = fma(lv[u], rv[j], acc[u][j]);
                    const uint32_t q2 = qq / (uint32_t)D;
                    m += (qq - q2 * (uint32_t)D) * (uint32_t)a.pw[s - 1];
                    qq = q2;
                }
#pragma unroll
                for (int u = 0; u < D; ++u)
#pragma unroll
                    for (int j = 0; j < V; ++j)
                        nxt[obase + u * dk1 + j] =
                            fma(c0v, (double)__ldg(node + obase + u * dk1 + j), acc[u][j]);
            }
            __syncthreads();
            double* t = cur;
            cur = nxt;
            nxt = t;
        }
        for (int64_t i = tid; i < a.T; i += blockDim.x) accq[i] = cur[i];
    }
}

// width -> last-letter block of the chain kernel (0: not available)
int chain_v(int width)
{
    switch (width) {
        case 2: return 2;
        case 3: return 3;
        case 4: return 4;
        case 5: return 5;
        case 6: return 3;
        case 8: return 2;
        default: return 0;
    }
}

template <typename TS>
using ChainFn = void (*)(ChainArgs);

template <typename TS>
ChainFn<TS> chain_fn(int width)
{
    switch (width) {
        case 2: return &chain_products_kernel<TS, 2, 2>;
        case 3: return &chain_products_kernel<TS, 3, 3>;
        case 4: return &chain_products_kernel<TS, 4, 4>;
        case 5: return &chain_products_kernel<TS, 5, 5>;
        case 6: return &chain_products_kernel<TS, 6, 3>;
        case 8: return &chain_products_kernel<TS, 8, 2>;
        default: return nullptr;
    }
}

constexpr int64_t kChainSmemLimit = 200 * 1024;

}  // namespace

bool chain_products_available(const Geometry& g)
{
    return g.depth >= 2 && chain_v(g.width) > 0 && 2 * g.size() * 8 <= kChainSmemLimit;
}

int chain_products(int src_mode, const Geometry& g, int64_t n, double* acc, const void* src,
                   const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                   cudaStream_t s)
{
    if (n == 0 || off[n] == 0) return RPYB_OK;
    if (!chain_products_available(g)) return fail(RPYB_E_UNSUPPORTED, "no chain kernel for this shape");
    const int V = chain_v(g.width);
    ChainArgs a;
    a.T = g.size();
    for (int k = 0; k <= kMaxDepth + 1; ++k) a.db[k] = g.db[k];
    for (int k = 0; k <= kMaxDepth; ++k) a.pw[k] = g.pw[k];
    int64_t u = 0;
    for (int k = 0; k <= kMaxDepth + 1; ++k) a.ucum[k] = 0;
    for (int k = 2; k <= g.depth; ++k) {
        a.ucum[k] = u;
        u += g.pw[k - 2] * (g.width / V);
    }
    for (int k = g.depth + 1; k <= kMaxDepth + 1; ++k) a.ucum[k] = u;
    a.utotal = u;
    a.depth = g.depth;
    a.n = n;
    // offsets and rows in one upload
    std::vector<int64_t> packed(off.begin(), off.begin() + n + 1);
    packed.insert(packed.end(), src_rows.begin(), src_rows.begin() + off[n]);
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    int rc;
    if ((rc = sc.get(packed.size() * 8, &mem))) return rc;
    int64_t* d = static_cast<int64_t*>(mem);
    if ((rc = upload_async(d, packed.data(), packed.size() * 8, s))) return rc;
    a.off = d;
    a.rows = d + n + 1;
    a.src = src;
    a.acc = acc;
    const size_t smem = (size_t)(2 * a.T * 8);
    const unsigned grid = (unsigned)std::min<int64_t>(n, 1 << 20);
    if (src_mode == RPYB_F64) {
        auto fn = chain_fn<double>(g.width);
        RPYB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fn<<<grid, kChainThreads, smem, s>>>(a);
    } else {
        auto fn = chain_fn<float>(g.width);
        RPYB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fn<<<grid, kChainThreads, smem, s>>>(a);
    }
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

int lie_maps_device(const Geometry& g, const LieMapsDev** out)
{
    static std::mutex mu;
    static LieMapsDev entries[128];
    static int n_entries = 0;
    int dev = 0;
    RPYB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    for (int i = 0; i < n_entries; ++i)
        if (entries[i].device == dev && entries[i].width == g.width && entries[i].depth == g.depth) {
            *out = &entries[i];
            return RPYB_OK;
        }
    if (n_entries == 128) return fail(RPYB_E_UNSUPPORTED, "too many cached Lie maps");
    const int64_t lie_dim = rpyb_lie_basis_size(g.width, g.depth);
    if (lie_dim < 0) return (int)lie_dim;
    LieMapsDev e;
    e.device = dev;
    e.width = g.width;
    e.depth = g.depth;
    e.lie_dim = lie_dim;
    int rc;
    if ((rc = upload_csr(g, 0, g.size(), &e.l2t_ptr, &e.l2t_idx, &e.l2t_val)) ||
        (rc = upload_csr(g, 1, lie_dim, &e.t2l_ptr, &e.t2l_idx, &e.t2l_val)))
        return rc;
    entries[n_entries] = e;
    *out = &entries[n_entries++];
    return RPYB_OK;
}

int unit_rows(int mode, void* out, int64_t ld, int64_t cols, const int64_t* idx, int64_t n,
              cudaStream_t s)
{
    if (n <= 0) return RPYB_OK;
    if (mode == RPYB_F64)
        unit_rows_kernel<double><<<grid_for(n * cols), 256, 0, s>>>(static_cast<double*>(out), ld,
                                                                    cols, idx, n);
    else
        unit_rows_kernel<float><<<grid_for(n * cols), 256, 0, s>>>(static_cast<float*>(out), ld,
                                                                   cols, idx, n);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

int ordered_products(int acc_mode, int src_mode, const Geometry& g, int64_t n, void* acc,
                     const void* src, const std::vector<int64_t>& off,
                     const std::vector<int64_t>& src_rows, cudaStream_t s)
{
    const int64_t T = g.size();
    if (n == 0) return RPYB_OK;
    const bool mixed = acc_mode == RPYB_F64 && src_mode == RPYB_F32;
    if (!mixed && acc_mode != src_mode) return fail(RPYB_E_INVALID, "unsupported dtype pair");
    // Rows sorted by factor count, most first: the rows still active at
    // position r are then a prefix of the order, and the products ping-pong
    // between two contiguous buffers without per-position scatters.
    std::vector<int64_t> order;
    order.reserve(n);
    for (int64_t q = 0; q < n; ++q)
        if (off[q + 1] > off[q]) order.push_back(q);
    const int64_t n1 = (int64_t)order.size();
    if (n1 == 0) return RPYB_OK;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
        return off[x + 1] - off[x] > off[y + 1] - off[y];
    });
    const int64_t maxc = off[order[0] + 1] - off[order[0]];
    // host index block: order (n1), final parity (n1), then per position r
    // the source rows of the m_r active rows
    std::vector<int64_t> packed(order);
    packed.reserve(2 * n1 + (size_t)off[n]);
    for (int64_t i = 0; i < n1; ++i) packed.push_back((off[order[i] + 1] - off[order[i]] - 1) & 1);
    std::vector<int64_t> pos(maxc + 1), active(maxc);
    for (int64_t r = 0; r < maxc; ++r) {
        pos[r] = (int64_t)packed.size();
        int64_t m = 0;
        while (m < n1 && off[order[m] + 1] - off[order[m]] > r) {
            packed.push_back(src_rows[off[order[m]] + r]);
            ++m;
        }
        active[r] = m;
    }
    const int64_t es = acc_mode == RPYB_F64 ? 8 : 4;
    const size_t idx_bytes = (packed.size() * 8 + 255) / 256 * 256;
    const size_t buf = (size_t)((n1 * T * es + 255) / 256 * 256);
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    int rc;
    if ((rc = sc.get(idx_bytes + 2 * buf, &mem))) return rc;
    int64_t* d_idx = static_cast<int64_t*>(mem);
    char* bufs[2] = {static_cast<char*>(mem) + idx_bytes, static_cast<char*>(mem) + idx_bytes + buf};
    if ((rc = upload_async(d_idx, packed.data(), packed.size() * 8, s))) return rc;
    for (int64_t r = 0; r < maxc; ++r) {
        const int64_t m = active[r];
        const void* lhs = (r == 0) ? acc : bufs[(r - 1) & 1];
        const int64_t* lhs_idx = (r == 0) ? d_idx : nullptr;   // gather by order at the start
        void* out = bufs[r & 1];
        const int64_t* rhs_idx = d_idx + pos[r];
        if (mixed)
            rc = rpyb_ft_mul_gather_mixed(g.width, g.depth, m, static_cast<double*>(out),
                                          static_cast<const double*>(lhs),
                                          static_cast<const float*>(src), T, nullptr, lhs_idx,
                                          rhs_idx, 0, s);
        else
            rc = rpyb_ft_mul_gather(acc_mode, g.width, g.depth, m, out, lhs, src, T, nullptr,
                                    lhs_idx, rhs_idx, 0, s);
        if (rc) return rc;
    }
    // rows back to their places: row i of the order ends in buffer parity[i]
    if (acc_mode == RPYB_F64)
        gather_final_kernel<double><<<grid_for(n1 * T), 256, 0, s>>>(
            static_cast<double*>(acc), reinterpret_cast<const double*>(bufs[0]),
            reinterpret_cast<const double*>(bufs[1]), T, d_idx, d_idx + n1, n1);
    else
        gather_final_kernel<float><<<grid_for(n1 * T), 256, 0, s>>>(
            static_cast<float*>(acc), reinterpret_cast<const float*>(bufs[0]),
            reinterpret_cast<const float*>(bufs[1]), T, d_idx, d_idx + n1, n1);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

size_t finish_scratch_bytes(const Geometry& g, int64_t lie_dim, int64_t n)
{
    n = std::max<int64_t>(n, 1);
    const int64_t log_ws = rpyb_ft_log_workspace_size(RPYB_F64, g.width, g.depth, n);
    const int64_t exp_ws = rpyb_ft_exp_workspace_size(RPYB_F64, g.width, g.depth, n);
    const size_t buf = (size_t)((n * g.size() * 8 + 255) / 256 * 256);
    const size_t lbuf = (size_t)((n * lie_dim * 8 + 255) / 256 * 256);
    return buf + lbuf + (size_t)std::max<int64_t>(std::max(log_ws, exp_ws), 1);
}

int finish_queries(const Geometry& g, const LieMapsDev& maps, int64_t m, double* acc,
                   double* out_logsig, int64_t ld_logsig, double* out_sig, int64_t ld_sig,
                   void* scratch, size_t scratch_bytes, cudaStream_t s)
{
    if (m <= 0) return RPYB_OK;
    const int64_t T = g.size(), L = maps.lie_dim;
    const size_t buf = (size_t)((m * T * 8 + 255) / 256 * 256);
    const size_t lbuf = (size_t)((m * L * 8 + 255) / 256 * 256);
    if (scratch_bytes < buf + lbuf + 1) return fail(RPYB_E_INVALID, "query scratch too small");
    double* tmp = static_cast<double*>(scratch);
    double* lie_tmp = reinterpret_cast<double*>(static_cast<char*>(scratch) + buf);
    void* ws = static_cast<char*>(scratch) + buf + lbuf;
    const size_t wsb = scratch_bytes - buf - lbuf;
    int rc;
    // log in float64 (its incoming out[0] must be zero), then tensor -> Lie
    RPYB_CUDA(cudaMemsetAsync(tmp, 0, (size_t)(m * T * 8), s));
    if ((rc = rpyb_ft_log(RPYB_F64, g.width, g.depth, m, tmp, acc, T, T, -1, -1, ws, wsb, s)))
        return rc;
    double* lie = out_logsig ? out_logsig : lie_tmp;
    const int64_t ld_lie = out_logsig ? ld_logsig : L;
    // the sparse map accumulates: clear its outputs first
    RPYB_CUDA(cudaMemset2DAsync(lie, (size_t)(ld_lie * 8), 0, (size_t)(L * 8), (size_t)m, s));
    if ((rc = rpyb_sparse_map(RPYB_F64, L, T, m, maps.t2l_ptr, maps.t2l_idx, maps.t2l_val, lie,
                              tmp, ld_lie, T, 1.0, s)))
        return rc;
    if (out_sig) {
        // algebra/src/context.cpp:156-159: exp(lie_to_tensor(log_signature))
        RPYB_CUDA(cudaMemsetAsync(tmp, 0, (size_t)(m * T * 8), s));
        if ((rc = rpyb_sparse_map(RPYB_F64, T, L, m, maps.l2t_ptr, maps.l2t_idx, maps.l2t_val, tmp,
                                  lie, T, ld_lie, 1.0, s)) ||
            (rc = rpyb_ft_exp(RPYB_F64, g.width, g.depth, m, out_sig, tmp, ld_sig, T, -1, ws, wsb,
                              s)))
            return rc;
    }
    return RPYB_OK;
}

int refine_and_dissect(int64_t n, const double* inf, const double* sup, double s0, double s1,
                       int32_t default_resolution, int32_t resolution, std::vector<int64_t>& k,
                       std::vector<int32_t>& p, std::vector<int64_t>& poff)
{
    const bool auto_res = resolution == RPYB_QUERY_RESOLUTION_AUTO;
    if (!auto_res && (resolution < -60 || resolution > 60))
        return fail(RPYB_E_INVALID, "query resolution out of range");
    k.clear();
    p.clear();
    k.reserve((size_t)n * 16);
    p.reserve((size_t)n * 16);
    poff.assign(n + 1, 0);
    int64_t kb[kMaxDyadicPieces];
    int32_t pb[kMaxDyadicPieces];
    for (int64_t q = 0; q < n; ++q) {
        double a = inf[q], b = sup[q];
        if (!(a <= b)) return fail(RPYB_E_INVALID, "inf must not be larger than sup");
        // trimmed to the support; empty queries keep no pieces
        const bool outside = b < s0 || a > s1;
        if (!outside) {
            a = std::max(a, s0);
            b = std::min(b, s1);
        }
        if (!outside && b - a != 0.0) {
            const int32_t tol =
                auto_res ? std::max<int32_t>(default_resolution, query_param_to_resolution(b - a) + 2)
                         : resolution;
            const int np = dissect_clopen(a, b, tol, kb, pb);
            if (np < 0) return np;
            k.insert(k.end(), kb, kb + np);
            p.insert(p.end(), pb, pb + np);
        }
        poff[q + 1] = (int64_t)k.size();
    }
    return RPYB_OK;
}

}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int rpyb_tensor_to_lie(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                                int64_t ld_out, const void* arg, int64_t ld_arg, void* stream)
{
    int rc;
    if (dtype != RPYB_F32 && dtype != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported dtype");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !arg) return fail(RPYB_E_INVALID, "null pointer");
    const int64_t L = rpyb_lie_basis_size(width, depth);
    if (L < 0) return (int)L;
    if (ld_out < L || ld_arg < g.size()) return fail(RPYB_E_INVALID, "row stride too small");
    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t es = dtype == RPYB_F64 ? 8 : 4;
    RPYB_CUDA(cudaMemset2DAsync(out, (size_t)ld_out * es, 0, (size_t)L * es, (size_t)batch, s));
    return rpyb_sparse_map(dtype, L, g.size(), batch, maps->t2l_ptr, maps->t2l_idx, maps->t2l_val,
                           out, arg, ld_out, ld_arg, 1.0, s);
}

RPYB_API int rpyb_lie_to_tensor(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                                int64_t ld_out, const void* arg, int64_t ld_arg, void* stream)
{
    int rc;
    if (dtype != RPYB_F32 && dtype != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported dtype");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !arg) return fail(RPYB_E_INVALID, "null pointer");
    const int64_t L = rpyb_lie_basis_size(width, depth);
    if (L < 0) return (int)L;
    if (ld_out < g.size() || ld_arg < L) return fail(RPYB_E_INVALID, "row stride too small");
    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t es = dtype == RPYB_F64 ? 8 : 4;
    RPYB_CUDA(cudaMemset2DAsync(out, (size_t)ld_out * es, 0, (size_t)g.size() * es, (size_t)batch,
                                s));
    return rpyb_sparse_map(dtype, g.size(), L, batch, maps->l2t_ptr, maps->l2t_idx, maps->l2t_val,
                           out, arg, ld_out, ld_arg, 1.0, s);
}

}  // extern "C"
