// Shared stream building blocks (see stream_ops.cuh).
#include <algorithm>
#include <map>
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

template <typename E>
int upload(const std::vector<E>& h, const E** out)
{
    E* d = nullptr;
    RPYB_CUDA(cudaMalloc(&d, std::max<size_t>(h.size(), 1) * sizeof(E)));
    if (!h.empty()) RPYB_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(E), cudaMemcpyHostToDevice));
    *out = d;
    return RPYB_OK;
}

// The packed form of a CSR map for lie_project_kernel: rows sorted by entry
// count (most first, stably) in groups of 32, each group padded to its
// longest row with zero entries and stored lane-interleaved (entry j of lane
// l at 32 j + l from the group's offset); an entry is 8 * column | value id
// << 19 (the byte offset of a float64 word of the row, so the kernel's
// gather needs no scaling).  False when a column does not fit 16 bits or
// the number of distinct values 13 bits.
bool pack_csr(const std::vector<int64_t>& hp, const std::vector<int64_t>& hi,
              const std::vector<double>& hv, int64_t n_rows, int64_t n_cols,
              std::vector<uint32_t>& goff, std::vector<uint32_t>& ent,
              std::vector<uint32_t>& perm, std::vector<double>& tab)
{
    if (n_cols > 0x10000) return false;
    std::map<uint64_t, uint32_t> ids;   // keyed by the value's bits
    tab.clear();
    auto id_of = [&](double v, uint32_t* out) {
        uint64_t bits;
        std::memcpy(&bits, &v, sizeof bits);
        auto it = ids.find(bits);
        if (it == ids.end()) {
            if (tab.size() > 0x1fff) return false;
            it = ids.emplace(bits, (uint32_t)tab.size()).first;
            tab.push_back(v);
        }
        *out = it->second;
        return true;
    };
    uint32_t zero_id = 0;
    if (!id_of(0.0, &zero_id)) return false;
    std::vector<int64_t> order(n_rows);
    for (int64_t r = 0; r < n_rows; ++r) order[r] = r;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
        return hp[x + 1] - hp[x] > hp[y + 1] - hp[y];
    });
    const int64_t groups = (n_rows + 31) / 32;
    goff.assign(groups + 1, 0);
    perm.assign(groups * 32, 0xffffffffu);
    ent.clear();
    for (int64_t g = 0; g < groups; ++g) {
        int64_t len = 0;
        for (int l = 0; l < 32 && g * 32 + l < n_rows; ++l) {
            const int64_t r = order[g * 32 + l];
            len = std::max<int64_t>(len, hp[r + 1] - hp[r]);
            perm[g * 32 + l] = (uint32_t)r;
        }
        for (int64_t j = 0; j < len; ++j)
            for (int l = 0; l < 32; ++l) {
                uint32_t e = zero_id << 19;
                if (g * 32 + l < n_rows) {
                    const int64_t r = order[g * 32 + l];
                    if (j < hp[r + 1] - hp[r]) {
                        const int64_t k = hp[r] + j;
                        uint32_t vid;
                        if (hi[k] < 0 || hi[k] >= n_cols || !id_of(hv[k], &vid)) return false;
                        e = ((uint32_t)hi[k] << 3) | (vid << 19);
                    }
                }
                ent.push_back(e);
            }
        if (ent.size() >= ((size_t)1 << 32)) return false;
        goff[g + 1] = (uint32_t)ent.size();
    }
    return true;
}

int upload_csr(const Geometry& g, int which, int64_t n_rows, const int64_t** ptr,
               const int64_t** idx, const double** val, LieMapsDev* packed_into = nullptr)
{
    const int64_t nnz = rpyb_lie_map_csr(g.width, g.depth, which, nullptr, nullptr, nullptr);
    if (nnz < 0) return (int)nnz;
    std::vector<int64_t> hp(n_rows + 1), hi(std::max<int64_t>(nnz, 1));
    std::vector<double> hv(std::max<int64_t>(nnz, 1));
    const int64_t got = rpyb_lie_map_csr(g.width, g.depth, which, hp.data(), hi.data(), hv.data());
    if (got < 0) return (int)got;
    if (packed_into) {
        std::vector<uint32_t> goff, ent, perm;
        std::vector<double> tab;
        if (pack_csr(hp, hi, hv, n_rows, g.size(), goff, ent, perm, tab)) {
            int rc;
            if ((rc = upload(goff, &packed_into->t2l_goff)) ||
                (rc = upload(ent, &packed_into->t2l_ent)) ||
                (rc = upload(perm, &packed_into->t2l_perm)) ||
                (rc = upload(tab, &packed_into->t2l_tab)))
                return rc;
            packed_into->t2l_slots = (int64_t)ent.size();
            packed_into->t2l_groups = (int64_t)goff.size() - 1;
            packed_into->t2l_ntab = (int64_t)tab.size();
        }
    }
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
// Tensor -> Lie projection with the packed map held in shared memory.  One
// persistent block per SM loads the map (column and value id per entry, the
// distinct values, the group offsets) once; for each of its rows of x it
// copies the row into shared memory with coalesced loads, and every warp
// computes groups of 32 Lie coordinates from shared memory, one per lane.
// The compact entries are what makes this pay: as (int64, float64) pairs the
// map is larger than a row of x and its gathers go to L2 for every row.  The
// lane-interleaved groups make a warp's entry reads consecutive words and
// give its lanes equal trip counts.
constexpr int kProjThreads = 1024;
constexpr int64_t kProjSmemLimit = 220 * 1024;

struct ProjArgs {
    int64_t n_cols = 0, slots = 0, groups = 0, ntab = 0, batch = 0;
    int64_t ld_y = 0, ld_x = 0;
    const uint32_t* goff = nullptr;
    const uint32_t* ent = nullptr;
    const uint32_t* perm = nullptr;
    const double* tab = nullptr;
};

template <typename T>
size_t proj_smem_bytes(const ProjArgs& a)
{
    const int64_t xs_bytes = (a.n_cols * (int64_t)sizeof(T) + 15) / 16 * 16;
    return (size_t)(xs_bytes + a.ntab * 8 + (a.groups + 1) * 4 + a.slots * 4);
}

template <typename T>
__global__ void __launch_bounds__(kProjThreads, 1)
lie_project_kernel(const ProjArgs a, T* __restrict__ y, const T* __restrict__ x)
{
    // the row first, so an entry's byte offset addresses its word directly
    extern __shared__ __align__(16) unsigned char proj_smem[];
    T* xs = reinterpret_cast<T*>(proj_smem);
    double* tab = reinterpret_cast<double*>(proj_smem + (a.n_cols * (int64_t)sizeof(T) + 15) / 16 * 16);
    uint32_t* goff = reinterpret_cast<uint32_t*>(tab + a.ntab);
    uint32_t* ent = goff + a.groups + 1;
    const int tid = (int)threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = (int)blockDim.x >> 5;
    for (int64_t i = tid; i < a.ntab; i += blockDim.x) tab[i] = a.tab[i];
    for (int64_t i = tid; i <= a.groups; i += blockDim.x) goff[i] = a.goff[i];
    for (int64_t i = tid; i < a.slots; i += blockDim.x) ent[i] = a.ent[i];
    constexpr int kU = 8;
    for (int64_t b = blockIdx.x; b < a.batch; b += gridDim.x) {
        __syncthreads();   // the map is loaded; the previous row's gathers are done
        const T* xr = x + b * a.ld_x;
        // eight independent loads in flight per thread
        for (int64_t c0 = tid; c0 < a.n_cols; c0 += kU * blockDim.x) {
            T v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int64_t c = c0 + (int64_t)u * blockDim.x;
                v[u] = c < a.n_cols ? __ldg(xr + c) : T(0);
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int64_t c = c0 + (int64_t)u * blockDim.x;
                if (c < a.n_cols) xs[c] = v[u];
            }
        }
        __syncthreads();
        if (b + gridDim.x < a.batch) {
            // the block's next row into L2 while this one is computed
            const char* nx = reinterpret_cast<const char*>(x + (b + gridDim.x) * a.ld_x);
            const int64_t bytes = a.n_cols * (int64_t)sizeof(T);
            for (int64_t l = (int64_t)tid * 128; l < bytes; l += (int64_t)blockDim.x * 128)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(nx + l));
        }
        T* yr = y + b * a.ld_y;
        for (int64_t g = warp; g < a.groups; g += nwarps) {
            double acc = 0.0;
            const uint32_t e1 = goff[g + 1];
#pragma unroll 4
            for (uint32_t k = goff[g] + lane; k < e1; k += 32) {
                const uint32_t w = ent[k];
                const uint32_t off = w & 0x7ffffu;   // 8 * column
                const T xv = *reinterpret_cast<const T*>(
                    proj_smem + (sizeof(T) == 8 ? off : off >> 1));
                acc = fma(tab[w >> 19], (double)xv, acc);
            }
            const uint32_t row = __ldg(a.perm + g * 32 + lane);
            if (row != 0xffffffffu) yr[row] = (T)acc;
        }
    }
}

template <typename T>
int launch_lie_project(const ProjArgs& a, void* y, const void* x, cudaStream_t s)
{
    const size_t smem = proj_smem_bytes<T>(a);
    RPYB_CUDA(cudaFuncSetAttribute(lie_project_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    const unsigned blocks = (unsigned)std::min<int64_t>(a.batch, 148);
    lie_project_kernel<T><<<blocks, kProjThreads, smem, s>>>(a, static_cast<T*>(y),
                                                             static_cast<const T*>(x));
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

// ------------------------------------------------------------------------
// Fused chain products: acc[q] <- src[r_0] * src[r_1] * ... (the unit for an
// empty list), or its float64 log, one block per row q, so that the running
// product never leaves the SM.  Its levels below the top are in shared
// memory (float64, double-buffered); its top level is spread over the
// threads' registers.  That split is exact: a top-level output word reads
// the lower levels of the left operand, the factor's words and only its own
// top-level word of the left operand (times the factor's scalar), so no
// thread needs another thread's top-level words.  A product is split like
// the blocked product kernel: a unit owns D first letters x V last letters
// of one middle part at a level k >= 2; levels 0 and 1 are done by the first
// threads.  Every thread owns TU top-level units (flat units tid, tid + B,
// ...); the lower units follow in the same flat order from the level below
// the top down, so the threads that take one more unit take a light one.
// The first factor is copied, not multiplied by the unit.  Factors are read
// from global memory (queries share them, so the popular ones stay in L2),
// and the next one is prefetched into L2 while a product runs.
struct ChainArgs {
    int64_t T = 0;
    int64_t db[kMaxDepth + 2] = {};
    int64_t pw[kMaxDepth + 1] = {};
    int64_t lo_begin[kMaxDepth + 2] = {};   // first lower unit of level k (2 <= k < depth)
    int64_t utop = 0, ulow = 0;             // top-level and lower units
    int depth = 0;
    int64_t n = 0;
    const int64_t* off = nullptr;      // [n + 1] into rows
    const int64_t* rows = nullptr;     // source row of each factor
    const void* src = nullptr;         // [*, T] factors (float or double)
    double* acc = nullptr;             // [n, T] out
    int log_out = 0;                   // write log(product) instead of the product
    void* dst = nullptr;               // instead of acc: rows dst_rows[q] of this
    const int64_t* dst_rows = nullptr; // [*, T] array of the factors' type
    // log_out with lie != null: the block projects its log onto the Hall
    // basis through the packed t2l map and writes lie[q * ld_lie + row]
    // instead of the log tensor
    double* lie = nullptr;
    int64_t ld_lie = 0, lie_dim = 0, pgroups = 0;
    const uint32_t* pgoff = nullptr;
    const uint32_t* pent = nullptr;
    const uint32_t* pperm = nullptr;
    const double* ptab = nullptr;
};

constexpr int kChainThreads = 512;

// out[D][V] (+)= sum over s = 1..k-1 of lhs level k-s (x) rhs level s at the
// unit (rp, c0) of level k: the left factor's D words of first letters u at
// middle part rp's prefix, the right factor's V words after it.  KC > 0 fixes
// k = KC at compile time; the loop is then unrolled, which lets the loads of
// all split points be issued together.
template <int D, int V, typename TR, bool GLOBAL_RHS, int KC = 0>
__device__ __forceinline__ void unit_splits(double (&acc)[D][V], const double* lhs, const TR* rhs,
                                            const ChainArgs& a, int k, uint32_t rp, int c0)
{
    uint32_t qq = rp;
    uint32_t m = 0;
    if constexpr (KC > 0) k = KC;
#pragma unroll
    for (int s = 1; s <= (KC > 0 ? KC : k) - 1; ++s) {
        const int p = k - s;
        double lv[D];
        double rv[V];
        const double* lp = lhs + a.db[p] + qq;
        const uint32_t dp1 = (uint32_t)a.pw[p - 1];
#pragma unroll
        for (int u = 0; u < D; ++u) lv[u] = lp[u * dp1];
        const TR* rq = rhs + a.db[s] + (int64_t)m * D + c0;
#pragma unroll
        for (int j = 0; j < V; ++j) {
            if constexpr (GLOBAL_RHS) rv[j] = (double)__ldg(rq + j);
            else rv[j] = (double)rq[j];
        }
#pragma unroll
        for (int u = 0; u < D; ++u)
#pragma unroll
            for (int j = 0; j < V; ++j) acc[u][j] = fma(lv[u], rv[j], acc[u][j]);
        const uint32_t q2 = qq / (uint32_t)D;
        m += (qq - q2 * (uint32_t)D) * (uint32_t)a.pw[s - 1];
        qq = q2;
    }
}

// the level and position of lower unit li (levels depth-1 down to 2)
template <int D, int V>
__device__ __forceinline__ void lower_unit(const ChainArgs& a, int64_t li, int& k, uint32_t& rp,
                                           int& c0, int64_t& obase, int64_t& dk1)
{
    constexpr int NB = D / V;
    k = a.depth - 1;
    while (k > 2 && li >= a.lo_begin[k - 1]) --k;
    const int64_t unit = li - a.lo_begin[k];
    rp = (uint32_t)(unit / NB);
    c0 = (int)(unit - (int64_t)rp * NB) * V;
    dk1 = a.pw[k - 1];
    obase = a.db[k] + (int64_t)rp * D + c0;
}

// NT > 0: the depth is NT (the top level's split loop is unrolled)
#ifndef RPYB_CHAIN_MIN_BLOCKS
#define RPYB_CHAIN_MIN_BLOCKS 1
#endif
template <typename TS, int D, int V, int TU, int NT>
__global__ void __launch_bounds__(kChainThreads, RPYB_CHAIN_MIN_BLOCKS)
chain_products_kernel(const ChainArgs a)
{
    constexpr int NB = D / V;
    extern __shared__ __align__(16) unsigned char chain_smem[];
    const int N = a.depth;
    const int64_t TL = a.db[N];   // words below the top level
    double* lo0 = reinterpret_cast<double*>(chain_smem);
    double* lo1 = lo0 + TL;
    const int tid = (int)threadIdx.x;
    const int B = (int)blockDim.x;
    const TS* src = static_cast<const TS*>(a.src);
    const int64_t tdk1 = a.pw[N - 1];
    // this thread's top-level units: output words tbase[t] + u * tdk1 + j
    int64_t tbase[TU];
    uint32_t trp[TU];
    int tc0[TU];
    bool town[TU];
#pragma unroll
    for (int t = 0; t < TU; ++t) {
        const int64_t f = tid + (int64_t)t * B;
        town[t] = f < a.utop;
        trp[t] = town[t] ? (uint32_t)(f / NB) : 0u;
        tc0[t] = town[t] ? (int)(f - (int64_t)trp[t] * NB) * V : 0;
        tbase[t] = a.db[N] + (int64_t)trp[t] * D + tc0[t];
    }
    int64_t f_low = tid;   // this thread's first lower unit (flat index)
    while (f_low < a.utop) f_low += B;

    for (int64_t q = blockIdx.x; q < a.n; q += gridDim.x) {
        const int64_t o0 = a.off[q], o1 = a.off[q + 1];
        double* accq = a.acc ? a.acc + q * a.T : nullptr;
        TS* dstq = a.dst ? static_cast<TS*>(a.dst) + a.dst_rows[q] * a.T : nullptr;
        if (o0 == o1 && a.lie) {   // the log of the unit: zero coordinates
            for (int64_t r = tid; r < a.lie_dim; r += B) a.lie[q * a.ld_lie + r] = 0.0;
            continue;
        }
        if (o0 == o1) {   // the unit, or its log
            for (int64_t i = tid; i < a.T; i += B) {
                const double v = (i == 0 && !a.log_out) ? 1.0 : 0.0;
                if (dstq) dstq[i] = (TS)v;
                else accq[i] = v;
            }
            continue;
        }
        double* cur = lo0;
        double* nxt = lo1;
        __syncthreads();   // the previous row's reads of the buffers are done
        const TS* first = src + a.rows[o0] * a.T;
        for (int64_t i = tid; i < TL; i += B) cur[i] = (double)__ldg(first + i);
        double top[TU][D][V];
#pragma unroll
        for (int t = 0; t < TU; ++t)
#pragma unroll
            for (int u = 0; u < D; ++u)
#pragma unroll
                for (int j = 0; j < V; ++j)
                    top[t][u][j] = town[t] ? (double)__ldg(first + tbase[t] + u * tdk1 + j) : 0.0;
        for (int64_t r = o0 + 1; r < o1; ++r) {
            __syncthreads();
            const TS* node = src + a.rows[r] * a.T;
            if (r + 1 < o1) {
                const char* nn = reinterpret_cast<const char*>(src + a.rows[r + 1] * a.T);
                const int64_t bytes = a.T * (int64_t)sizeof(TS);
                for (int64_t l = (int64_t)tid * 128; l < bytes; l += (int64_t)B * 128)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(nn + l));
            }
            const double node0 = (double)__ldg(node);
            const double c0v = cur[0];
            if (tid == 0) nxt[0] = c0v * node0;
            if (tid < D) nxt[1 + tid] = cur[1 + tid] * node0 + c0v * (double)__ldg(node + 1 + tid);
            // top-level units, in registers
#pragma unroll
            for (int t = 0; t < TU; ++t) {
                if (!town[t]) continue;
#pragma unroll
                for (int u = 0; u < D; ++u)
#pragma unroll
                    for (int j = 0; j < V; ++j) top[t][u][j] *= node0;
                unit_splits<D, V, TS, true, NT>(top[t], cur, node, a, N, trp[t], tc0[t]);
#pragma unroll
                for (int u = 0; u < D; ++u)
#pragma unroll
                    for (int j = 0; j < V; ++j)
                        top[t][u][j] =
                            fma(c0v, (double)__ldg(node + tbase[t] + u * tdk1 + j), top[t][u][j]);
            }
            // lower units, in shared memory
            for (int64_t f = f_low; f < a.utop + a.ulow; f += B) {
                int k, c0;
                uint32_t rp;
                int64_t obase, dk1;
                lower_unit<D, V>(a, f - a.utop, k, rp, c0, obase, dk1);
                double acc[D][V];
#pragma unroll
                for (int u = 0; u < D; ++u)
#pragma unroll
                    for (int j = 0; j < V; ++j) acc[u][j] = cur[obase + u * dk1 + j] * node0;
                unit_splits<D, V, TS, true>(acc, cur, node, a, k, rp, c0);
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
        if (a.log_out) {
            // log(X) of the product X by the Horner steps of the float64 log
            // (free_tensor_log.hpp:23-38): with Y = X - X_0 and R = 0, for
            // deg = N down to 1, R <- (R + c_deg) Y truncated to the levels
            // N - deg + 1 and below, c_deg = (-1)^(deg+1) / deg.  Y's lower
            // levels stay in `cur`, its top level in `top`; R's lower levels
            // ping-pong between `nxt` and a third buffer.  R's top level is
            // formed only in the last step, in place of Y's own top words.
            double* rc = nxt;
            double* rn = lo0 + 2 * TL;   // the third buffer
            for (int s = 1; s <= N; ++s) {
                const int deg = N - s + 1;
                const double c = (deg % 2 == 0) ? -1.0 / (double)deg : 1.0 / (double)deg;
                __syncthreads();   // R's previous step (and Y) complete
                if (tid < D) rn[1 + tid] = c * cur[1 + tid];
                if (s == N) {
#pragma unroll
                    for (int t = 0; t < TU; ++t) {
                        if (!town[t]) continue;
#pragma unroll
                        for (int u = 0; u < D; ++u)
#pragma unroll
                            for (int j = 0; j < V; ++j) top[t][u][j] *= c;
                        unit_splits<D, V, double, false, NT>(top[t], rc, cur, a, N, trp[t],
                                                             tc0[t]);
                    }
                }
                for (int64_t f = f_low; f < a.utop + a.ulow; f += B) {
                    int k, c0;
                    uint32_t rp;
                    int64_t obase, dk1;
                    lower_unit<D, V>(a, f - a.utop, k, rp, c0, obase, dk1);
                    if (k > s) continue;
                    double acc[D][V];
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j) acc[u][j] = c * cur[obase + u * dk1 + j];
                    unit_splits<D, V, double, false>(acc, rc, cur, a, k, rp, c0);
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j) rn[obase + u * dk1 + j] = acc[u][j];
                }
                double* t = rc;
                rc = rn;
                rn = t;
            }
            __syncthreads();
            if (tid == 0) rc[0] = 0.0;
            __syncthreads();
            cur = rc;
        }
        if (a.lie) {
            // the whole log into shared memory (after the three log
            // buffers), then one warp per group of 32 Lie rows; an entry is
            // 8 * column | value id << 19 (see pack_csr)
            double* xs = lo0 + 3 * TL;
            for (int64_t i = tid; i < TL; i += B) xs[i] = cur[i];
#pragma unroll
            for (int t = 0; t < TU; ++t)
                if (town[t])
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j) xs[tbase[t] + u * tdk1 + j] = top[t][u][j];
            __syncthreads();
            const unsigned char* xb = reinterpret_cast<const unsigned char*>(xs);
            const int lane = tid & 31, nw = B >> 5;
            double* yq = a.lie + q * a.ld_lie;
            for (int64_t gi = tid >> 5; gi < a.pgroups; gi += nw) {
                double accp = 0.0;
                const uint32_t e1 = __ldg(a.pgoff + gi + 1);
#pragma unroll 4
                for (uint32_t k = __ldg(a.pgoff + gi) + lane; k < e1; k += 32) {
                    const uint32_t w = __ldg(a.pent + k);
                    accp = fma(__ldg(a.ptab + (w >> 19)),
                               *reinterpret_cast<const double*>(xb + (w & 0x7ffffu)), accp);
                }
                const uint32_t row = __ldg(a.pperm + gi * 32 + lane);
                if (row != 0xffffffffu) yq[row] = accp;
            }
            continue;
        }
        if (dstq) {
            // straight into the factors' array, rounded once to its type
            for (int64_t i = tid; i < TL; i += B) dstq[i] = (TS)cur[i];
#pragma unroll
            for (int t = 0; t < TU; ++t)
                if (town[t])
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j) dstq[tbase[t] + u * tdk1 + j] = (TS)top[t][u][j];
        } else {
            for (int64_t i = tid; i < TL; i += B) accq[i] = cur[i];
#pragma unroll
            for (int t = 0; t < TU; ++t)
                if (town[t])
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j) accq[tbase[t] + u * tdk1 + j] = top[t][u][j];
        }
    }
}

// width -> last-letter block of the chain kernel (0: not available)
int chain_v(int width)
{
    switch (width) {
        case 2: return 2;
        case 3: return 3;
        case 4: return 4;
        case 5: return 1;
        case 6: return 3;
        case 8: return 2;
        default: return 0;
    }
}

// top-level units a thread holds in registers (0: the shape is not
// covered); two only where two units' words fit the registers unspilled
int chain_tu(const Geometry& g)
{
    const int V = chain_v(g.width);
    if (V == 0 || g.depth < 2) return 0;
    const int64_t utop = g.pw[g.depth - 2] * (g.width / V);
    const int64_t tu = (utop + kChainThreads - 1) / kChainThreads;
    if (tu == 1) return 1;
    if (tu == 2 && g.width <= 3) return 2;
    return 0;
}

using ChainFn = void (*)(ChainArgs);

template <typename TS, int NT>
ChainFn chain_fn_nt(int width, int tu)
{
    if (tu == 2) {
        switch (width) {
            case 2: return &chain_products_kernel<TS, 2, 2, 2, NT>;
            case 3: return &chain_products_kernel<TS, 3, 3, 2, NT>;
            default: return nullptr;
        }
    }
    switch (width) {
        case 2: return &chain_products_kernel<TS, 2, 2, 1, NT>;
        case 3: return &chain_products_kernel<TS, 3, 3, 1, NT>;
        case 4: return &chain_products_kernel<TS, 4, 4, 1, NT>;
        case 5: return &chain_products_kernel<TS, 5, 1, 1, NT>;
        case 6: return &chain_products_kernel<TS, 6, 3, 1, NT>;
        case 8: return &chain_products_kernel<TS, 8, 2, 1, NT>;
        default: return nullptr;
    }
}

// depths 5 and 6 get a kernel with the top level's split loop unrolled
template <typename TS>
ChainFn chain_fn(int width, int depth, int tu)
{
    if (depth == 5) return chain_fn_nt<TS, 5>(width, tu);
    if (depth == 6) return chain_fn_nt<TS, 6>(width, tu);
    return chain_fn_nt<TS, 0>(width, tu);
}

constexpr int64_t kChainSmemLimit = 200 * 1024;

}  // namespace

bool chain_products_available(const Geometry& g)
{
    return chain_tu(g) > 0 && 3 * g.db[g.depth] * 8 <= kChainSmemLimit;
}

static int chain_launch(int src_mode, const Geometry& g, int64_t n, double* acc, const void* src,
                        const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                        bool log_out, void* dst, const std::vector<int64_t>* dst_rows,
                        cudaStream_t s, const LieMapsDev* maps = nullptr, double* lie = nullptr,
                        int64_t ld_lie = 0);

int chain_products(int src_mode, const Geometry& g, int64_t n, double* acc, const void* src,
                   const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                   bool log_out, cudaStream_t s)
{
    return chain_launch(src_mode, g, n, acc, src, off, src_rows, log_out, nullptr, nullptr, s);
}

int chain_products_into(int src_mode, const Geometry& g, int64_t n, void* nodes,
                        const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                        const std::vector<int64_t>& dst_rows, cudaStream_t s)
{
    return chain_launch(src_mode, g, n, nullptr, nodes, off, src_rows, false, nodes, &dst_rows, s);
}

bool chain_lie_available(const Geometry& g, const LieMapsDev& maps)
{
    return chain_products_available(g) && maps.t2l_ent &&
           (size_t)(3 * g.db[g.depth] + g.size()) * 8 <= (size_t)kChainSmemLimit;
}

int chain_products_lie(int src_mode, const Geometry& g, int64_t n, const void* src,
                       const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                       const LieMapsDev& maps, double* lie, int64_t ld_lie, cudaStream_t s)
{
    if (!chain_lie_available(g, maps)) return fail(RPYB_E_UNSUPPORTED, "no fused projection for this shape");
    return chain_launch(src_mode, g, n, nullptr, src, off, src_rows, true, nullptr, nullptr, s,
                        &maps, lie, ld_lie);
}

static int chain_launch(int src_mode, const Geometry& g, int64_t n, double* acc, const void* src,
                        const std::vector<int64_t>& off, const std::vector<int64_t>& src_rows,
                        bool log_out, void* dst, const std::vector<int64_t>* dst_rows,
                        cudaStream_t s, const LieMapsDev* maps, double* lie, int64_t ld_lie)
{
    if (n == 0) return RPYB_OK;
    if (!chain_products_available(g)) return fail(RPYB_E_UNSUPPORTED, "no chain kernel for this shape");
    if (off[n] == 0 && lie) {
        RPYB_CUDA(cudaMemset2DAsync(lie, (size_t)ld_lie * 8, 0, (size_t)maps->lie_dim * 8,
                                    (size_t)n, s));
        return RPYB_OK;
    }
    if (off[n] == 0 && !dst) {
        if (log_out) {
            RPYB_CUDA(cudaMemsetAsync(acc, 0, (size_t)(n * g.size() * 8), s));
            return RPYB_OK;
        }
        return unit_rows(RPYB_F64, acc, g.size(), g.size(), nullptr, n, s);
    }
    const int V = chain_v(g.width), NB = g.width / V, tu = chain_tu(g);
    ChainArgs a;
    a.T = g.size();
    for (int k = 0; k <= kMaxDepth + 1; ++k) a.db[k] = g.db[k];
    for (int k = 0; k <= kMaxDepth; ++k) a.pw[k] = g.pw[k];
    a.utop = g.pw[g.depth - 2] * NB;
    // lower levels depth-1 down to 2, in that order
    int64_t u = 0;
    for (int k = g.depth - 1; k >= 2; --k) {
        a.lo_begin[k] = u;
        u += g.pw[k - 2] * NB;
    }
    a.lo_begin[1] = u;
    a.ulow = u;
    a.depth = g.depth;
    a.n = n;
    // offsets and rows in one upload
    std::vector<int64_t> packed(off.begin(), off.begin() + n + 1);
    packed.insert(packed.end(), src_rows.begin(), src_rows.begin() + off[n]);
    if (dst) packed.insert(packed.end(), dst_rows->begin(), dst_rows->begin() + n);
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
    a.log_out = log_out ? 1 : 0;
    a.dst = dst;
    a.dst_rows = dst ? d + n + 1 + off[n] : nullptr;
    if (lie) {
        a.lie = lie;
        a.ld_lie = ld_lie;
        a.lie_dim = maps->lie_dim;
        a.pgroups = maps->t2l_groups;
        a.pgoff = maps->t2l_goff;
        a.pent = maps->t2l_ent;
        a.pperm = maps->t2l_perm;
        a.ptab = maps->t2l_tab;
    }
    const size_t smem =
        (size_t)((log_out ? 3 : 2) * g.db[g.depth] * 8) + (lie ? (size_t)g.size() * 8 : 0);
    const unsigned grid = (unsigned)std::min<int64_t>(n, 1 << 20);
    ChainFn fn = src_mode == RPYB_F64 ? chain_fn<double>(g.width, g.depth, tu)
                                      : chain_fn<float>(g.width, g.depth, tu);
    if (smem > 48 * 1024)
        RPYB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    fn<<<grid, kChainThreads, smem, s>>>(a);
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
        (rc = upload_csr(g, 1, lie_dim, &e.t2l_ptr, &e.t2l_idx, &e.t2l_val, &e)))
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

int lie_project(int dtype, const Geometry& g, const LieMapsDev& maps, int64_t m, void* lie,
                int64_t ld_lie, const void* x, int64_t ld_x, cudaStream_t s)
{
    if (m <= 0) return RPYB_OK;
    const int64_t T = g.size(), L = maps.lie_dim;
    ProjArgs a;
    a.n_cols = T;
    a.slots = maps.t2l_slots;
    a.groups = maps.t2l_groups;
    a.ntab = maps.t2l_ntab;
    a.batch = m;
    a.ld_y = ld_lie;
    a.ld_x = ld_x;
    a.goff = maps.t2l_goff;
    a.ent = maps.t2l_ent;
    a.perm = maps.t2l_perm;
    a.tab = maps.t2l_tab;
    if (maps.t2l_ent) {
        if (dtype == RPYB_F64 && proj_smem_bytes<double>(a) <= (size_t)kProjSmemLimit)
            return launch_lie_project<double>(a, lie, x, s);
        if (dtype == RPYB_F32 && proj_smem_bytes<float>(a) <= (size_t)kProjSmemLimit)
            return launch_lie_project<float>(a, lie, x, s);
    }
    // the sparse map accumulates: clear its outputs first
    const size_t es = dtype == RPYB_F64 ? 8 : 4;
    RPYB_CUDA(cudaMemset2DAsync(lie, (size_t)ld_lie * es, 0, (size_t)L * es, (size_t)m, s));
    return rpyb_sparse_map(dtype, L, T, m, maps.t2l_ptr, maps.t2l_idx, maps.t2l_val, lie, x, ld_lie,
                           ld_x, 1.0, s);
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

double* finish_lie_rows(const Geometry& g, int64_t lie_dim, int64_t m, void* scratch,
                        double* out_logsig, int64_t ld_logsig, int64_t* ld_lie)
{
    (void)lie_dim;
    *ld_lie = out_logsig ? ld_logsig : lie_dim;
    if (out_logsig) return out_logsig;
    const size_t buf = (size_t)((m * g.size() * 8 + 255) / 256 * 256);
    return reinterpret_cast<double*>(static_cast<char*>(scratch) + buf);
}

int finish_queries(const Geometry& g, const LieMapsDev& maps, int64_t m, double* acc,
                   bool acc_is_log, double* out_logsig, int64_t ld_logsig, double* out_sig,
                   int64_t ld_sig, void* scratch, size_t scratch_bytes, cudaStream_t s,
                   bool lie_ready)
{
    if (m <= 0) return RPYB_OK;
    const int64_t T = g.size(), L = maps.lie_dim;
    const size_t buf = (size_t)((m * T * 8 + 255) / 256 * 256);
    const size_t lbuf = (size_t)((m * L * 8 + 255) / 256 * 256);
    if (scratch_bytes < buf + lbuf + 1) return fail(RPYB_E_INVALID, "query scratch too small");
    double* tmp = static_cast<double*>(scratch);
    void* ws = static_cast<char*>(scratch) + buf + lbuf;
    const size_t wsb = scratch_bytes - buf - lbuf;
    int rc;
    int64_t ld_lie = 0;
    double* lie = finish_lie_rows(g, L, m, scratch, out_logsig, ld_logsig, &ld_lie);
    if (!lie_ready) {
        // log in float64 (its incoming out[0] must be zero), then tensor -> Lie
        const double* logt = acc;
        if (!acc_is_log) {
            RPYB_CUDA(cudaMemsetAsync(tmp, 0, (size_t)(m * T * 8), s));
            if ((rc = rpyb_ft_log(RPYB_F64, g.width, g.depth, m, tmp, acc, T, T, -1, -1, ws, wsb,
                                  s)))
                return rc;
            logt = tmp;
        }
        if ((rc = lie_project(RPYB_F64, g, maps, m, lie, ld_lie, logt, T, s))) return rc;
    }
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
    return lie_project(dtype, g, *maps, batch, out, ld_out, arg, ld_arg,
                       static_cast<cudaStream_t>(stream));
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
