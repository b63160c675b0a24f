// Batched truncated free-tensor product kernels (sm_100a).
//
// Work decomposition.  Output level k (k >= 1) holds d^k words; write a word
// as w = u * d^(k-1) + r with u its first letter.  For every split p >= 1 the
// right factor R_{k-p}[w mod d^(k-p)] = R_{k-p}[r mod d^(k-p)] does not depend
// on u.  The suffix kernel (product_kernel) lets one thread own a suffix r and
// produce the d words {u * d^(k-1) + r : u < d}; the blocked kernels (widths
// 2..6 and 8, the default) let a thread own the d first letters times a block
// of last letters, so that a split point's left words are shared by the
// block and its right words by the first letters.  The top-level streams
// (L_k, R_k, old out_k) are coalesced across consecutive units.  The (level,
// unit) pairs of all output levels are flattened into one index space that
// is cut into tiles; blockIdx.x walks tiles of one row so that a row's lower
// levels stay hot in L2, blockIdx.y walks rows.  Float64 rows of width 2
// take their levels >= 8 from a kernel whose 32 lanes own the last five
// letters of a word instead (product_kernel_w2: every load one coalesced
// request or one broadcast).
//
// Arithmetic.  float64: the terms are added in the reference order (lhs
// degree from high to low, free_tensor_fma.hpp:31-46) with FMA.  float32: by
// default every product of two float32 words (exact in float64) is
// accumulated in float64 and rounded once; a double-float pair or plain
// float32 accumulation can be selected (RPYB_F32_ACC).
#include "product.cuh"

#include <algorithm>
#include <cstdlib>

namespace rpyb {
namespace {

constexpr int kThreads = 256;

struct KArgs {
    int width;
    int klo, khi;
    int64_t db[kMaxDepth + 2];
    int64_t pw[kMaxDepth + 1];
    int64_t fcum[kMaxDepth + 2];   // fcum[k] = sum_{j<k, j>=klo} d^(j-1)
    int pmin[kMaxDepth + 1], pmax[kMaxDepth + 1];
    double scale[kMaxDepth + 1];
    int64_t ftotal;
    int64_t tile_r;
    bool accumulate, lhs0_from_mem;
    double lhs0_add;
    bool l0_write, l0_prod;
    int l0_base;
    double l0_const, scale0;
    void* out;
    const void* lhs;
    const void* rhs;
    const void* addend;
    int64_t ld_out, ld_lhs, ld_rhs, ld_add;
    const int64_t* out_idx;
    const int64_t* lhs_idx;
    const int64_t* rhs_idx;
    int64_t batch;
    bool prefetch;   // L2 prefetch of the p = 0 term's streamed right words
    int sklo, skhi;  // blocked kernels: levels computed word by word by each
                     // row's first tile (with the level-0 rule); none if skhi < sklo
};

__device__ __forceinline__ void prefetch_l2(const void* p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <typename T>
struct Acc;

template <>
struct Acc<double> {
    double v;
    __device__ __forceinline__ void init(double x) { v = x; }
    __device__ __forceinline__ void add(double a, double b) { v = fma(a, b, v); }
    __device__ __forceinline__ double value() const { return v; }
};

template <>
struct Acc<float> {
    DF v;
    __device__ __forceinline__ void init(float x) { v.hi = x; v.lo = 0.f; }
    __device__ __forceinline__ void add(float a, float b) { df_add_prod(v, a, b); }
    __device__ __forceinline__ float value() const { return df_value(v); }
};

// float32 accumulators.  The default accumulates the exact float32 products
// in float64 (one conversion and one FP64 FMA per product; 53 significant
// bits, more than the double-float pair above, and faster on B200).
// RPYB_F32_ACC selects the double-float pair ("df") or plain float32 FMAs
// ("plain") for comparison.
struct AccF32in64 {
    double v;
    __device__ __forceinline__ void init(float x) { v = (double)x; }
    __device__ __forceinline__ void add(float a, float b) { v = fma((double)a, (double)b, v); }
    __device__ __forceinline__ float value() const { return (float)v; }
};
struct AccF32Plain {
    float v;
    __device__ __forceinline__ void init(float x) { v = x; }
    __device__ __forceinline__ void add(float a, float b) { v = fmaf(a, b, v); }
    __device__ __forceinline__ float value() const { return v; }
};

template <typename T, int MODE>
struct AccSel {
    using type = Acc<T>;
};
template <>
struct AccSel<float, 1> {
    using type = AccF32in64;
};
template <>
struct AccSel<float, 2> {
    using type = AccF32Plain;
};

// T: output, left factor and accumulation type; TR: right factor type
// (TR = float with T = double is the mixed mode: float32 right factors
// accumulated into float64 rows).
template <typename T, typename TR, int D, int ACC = 0>
__global__ void __launch_bounds__(kThreads)
product_kernel(const KArgs a)
{
    const int d = (D > 0) ? D : a.width;
    const int64_t f_begin = (int64_t)blockIdx.x * a.tile_r;
    const int64_t f_end = min(f_begin + a.tile_r, a.ftotal);

    for (int64_t b = blockIdx.y; b < a.batch; b += gridDim.y) {
        const int64_t ro = a.out_idx ? a.out_idx[b] : b;
        const int64_t rl = a.lhs_idx ? a.lhs_idx[b] : b;
        const int64_t rr = a.rhs_idx ? a.rhs_idx[b] : b;
        T* __restrict__ out = static_cast<T*>(a.out) + ro * a.ld_out;
        const T* __restrict__ lhs = static_cast<const T*>(a.lhs) + rl * a.ld_lhs;
        const TR* __restrict__ rhs = static_cast<const TR*>(a.rhs) + rr * a.ld_rhs;
        const T* __restrict__ add =
            a.addend ? static_cast<const T*>(a.addend) + ro * a.ld_add : nullptr;

        const T lhs0 = (a.lhs0_from_mem ? __ldg(lhs) : T(0)) + T(a.lhs0_add);

        if (a.l0_write && blockIdx.x == 0 && threadIdx.x == 0) {
            T v0 = T(0);
            if (a.l0_base == 1) v0 = out[0];
            else if (a.l0_base == 2) v0 = add[0];
            v0 += T(a.l0_const);
            if (a.l0_prod) v0 += T(a.scale0) * (lhs0 * T(__ldg(rhs)));
            out[0] = v0;
        }

        for (int64_t f = f_begin + threadIdx.x; f < f_end; f += kThreads) {
            int k = a.klo;
            while (f >= a.fcum[k + 1]) ++k;
            const int64_t r = f - a.fcum[k];
            const int64_t dk1 = a.pw[k - 1];
            const int64_t obase = a.db[k] + r;

            typename AccSel<T, ACC>::type acc[(D > 0) ? D : 16];
#pragma unroll
            for (int u = 0; u < ((D > 0) ? D : 16); ++u) {
                if (D > 0 || u < d) {
                    acc[u].init(a.accumulate ? out[obase + u * dk1] : T(0));
                }
            }

            const int pmax = a.pmax[k];
            const int pmin = a.pmin[k];
            if (pmax >= pmin) {
                // Walk the split points from p = k down (suffix length s = k - p
                // growing), peeling one letter off the prefix q onto the suffix m
                // per step; word indices fit in 32 bits, and with a compile-time
                // width the division by d is a multiply-shift.
                uint32_t q = (uint32_t)r;
                uint32_t m = 0;
                int s = 0;
                for (int p = k; p >= pmin; --p) {
                    if (p <= pmax) {
                        if (p == 0) {
                            const TR* rk = rhs + a.db[k] + r;
#pragma unroll
                            for (int u = 0; u < ((D > 0) ? D : 16); ++u) {
                                if (D > 0 || u < d) acc[u].add(lhs0, T(__ldg(rk + u * dk1)));
                            }
                        } else {
                            const T rv = T(__ldg(rhs + a.db[s] + m));
                            const T* lp = lhs + a.db[p] + q;
                            const uint32_t dp1 = (uint32_t)a.pw[p - 1];
#pragma unroll
                            for (int u = 0; u < ((D > 0) ? D : 16); ++u) {
                                if (D > 0 || u < d) acc[u].add(__ldg(lp + u * dp1), rv);
                            }
                        }
                    }
                    // advance to suffix length s + 1
                    const uint32_t q2 = (D > 0) ? q / (uint32_t)D : q / (uint32_t)d;
                    m += (q - q2 * (uint32_t)d) * (uint32_t)a.pw[s];
                    q = q2;
                    ++s;
                }
            }

            const T sc = T(a.scale[k]);
#pragma unroll
            for (int u = 0; u < ((D > 0) ? D : 16); ++u) {
                if (D > 0 || u < d) {
                    const int64_t o = obase + u * dk1;
                    T v;
                    if (a.accumulate) {
                        v = acc[u].value();
                    } else {
                        v = sc * acc[u].value();
                        if (add) v += add[o];
                    }
                    out[o] = v;
                }
            }
        }
    }
}

// Levels sklo..skhi (at most the owned letters) and the level-0 rule of one
// row, word by word, by the threads of the row's first tile: the same terms
// in the same order as product_kernel, so the blocked kernels need no
// second launch for them.
template <typename T, typename TR, typename AccT, bool POW2 = false>
__device__ __forceinline__ void small_levels(const KArgs& a, T* __restrict__ out,
                                             const T* __restrict__ lhs,
                                             const TR* __restrict__ rhs,
                                             const T* __restrict__ add, T lhs0)
{
    if (a.l0_write && threadIdx.x == 0) {
        T v0 = T(0);
        if (a.l0_base == 1) v0 = out[0];
        else if (a.l0_base == 2) v0 = add[0];
        v0 += T(a.l0_const);
        if (a.l0_prod) v0 += T(a.scale0) * (lhs0 * T(__ldg(rhs)));
        out[0] = v0;
    }
    int64_t w = threadIdx.x;
    for (int k = a.sklo; k <= a.skhi; ++k) {
        const int64_t nk = a.pw[k];
        for (; w < nk; w += kThreads) {
            const int64_t o = a.db[k] + w;
            AccT acc;
            acc.init(a.accumulate ? out[o] : T(0));
            for (int p = k; p >= a.pmin[k]; --p) {
                if (p > a.pmax[k]) continue;
                const int sdeg = k - p;
                const int64_t ds = a.pw[sdeg];
                int64_t li, ri;
                if constexpr (POW2) {
                    // width 2: ds = 2^sdeg
                    li = w >> sdeg;
                    ri = w & (ds - 1);
                } else {
                    li = w / ds;
                    ri = w - li * ds;
                }
                const T lv = (p == 0) ? lhs0 : __ldg(lhs + a.db[p] + li);
                acc.add(lv, T(__ldg(rhs + a.db[sdeg] + ri)));
            }
            T v;
            if (a.accumulate) {
                v = acc.value();
            } else {
                v = T(a.scale[k]) * acc.value();
                if (add) v += add[o];
            }
            out[o] = v;
        }
        w -= nk;
    }
}

// Blocked variant for output levels k >= 2 (one owned last letter).  A thread owns the D x V words
//   u d^(k-1) + r' d + c0 + j    (u < D first letters, j < V last letters)
// for one middle part r' (k-2 letters) and one block c0 .. c0+V-1 of last
// letters.  For a split point 1 <= p <= k-1 the D left-factor words
// (u, r'_1 .. r'_{p-1}) do not depend on the last letter and the V
// right-factor words (r'_{p..k-2}, c) do not depend on the first, so D + V
// loads feed D V FMAs; the top-level words of the p = k and p = 0 terms are
// read as runs of V consecutive words.
template <typename T, typename TR, int D, int V, int ACC = 0, int MINB = 1, bool PIPE = false>
__global__ void __launch_bounds__(kThreads, MINB)
product_kernel_blocked(const KArgs a)
{
    constexpr int NB = D / V;
    using AccT = typename AccSel<T, ACC>::type;
    const int64_t f_begin = (int64_t)blockIdx.x * a.tile_r;
    const int64_t f_end = min(f_begin + a.tile_r, a.ftotal);

    for (int64_t b = blockIdx.y; b < a.batch; b += gridDim.y) {
        const int64_t ro = a.out_idx ? a.out_idx[b] : b;
        const int64_t rl = a.lhs_idx ? a.lhs_idx[b] : b;
        const int64_t rr = a.rhs_idx ? a.rhs_idx[b] : b;
        T* __restrict__ out = static_cast<T*>(a.out) + ro * a.ld_out;
        const T* __restrict__ lhs = static_cast<const T*>(a.lhs) + rl * a.ld_lhs;
        const TR* __restrict__ rhs = static_cast<const TR*>(a.rhs) + rr * a.ld_rhs;
        const T* __restrict__ add =
            a.addend ? static_cast<const T*>(a.addend) + ro * a.ld_add : nullptr;
        const T lhs0 = (a.lhs0_from_mem ? __ldg(lhs) : T(0)) + T(a.lhs0_add);
        const T rhs0 = T(__ldg(rhs));
        if (blockIdx.x == 0) small_levels<T, TR, AccT>(a, out, lhs, rhs, add, lhs0);

        for (int64_t f = f_begin + threadIdx.x; f < f_end; f += kThreads) {
            int k = a.klo;
            while (f >= a.fcum[k + 1]) ++k;
            const int64_t unit = f - a.fcum[k];
            const uint32_t rp = (uint32_t)(unit / NB);
            const int c0 = (int)(unit - (int64_t)rp * NB) * V;
            const int64_t dk1 = a.pw[k - 1];
            const int64_t obase = a.db[k] + (int64_t)rp * D + c0;
            // the p = 0 term's right words are read last: start them towards L2 now
            if (a.prefetch && a.pmin[k] <= 0 && a.pmax[k] >= 0) {
#pragma unroll
                for (int u = 0; u < D; ++u) prefetch_l2(rhs + obase + u * dk1);
            }

            AccT acc[D][V];
#pragma unroll
            for (int u = 0; u < D; ++u)
#pragma unroll
                for (int j = 0; j < V; ++j)
                    acc[u][j].init(a.accumulate ? out[obase + u * dk1 + j] : T(0));

            const int pmax = a.pmax[k];
            const int pmin = a.pmin[k];
            if (pmax >= pmin) {
                if (k <= pmax && k >= pmin) {
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j)
                            acc[u][j].add(__ldg(lhs + obase + u * dk1 + j), rhs0);
                }
                // split p = k - s: left word (u, r'_1..r'_{p-1}) = u d^(p-1) + q,
                // right word (r'_p..r'_{k-2}, c) = m d + c with q, m peeled from r'
                uint32_t q = rp;
                uint32_t m = 0;
                if (PIPE && pmin <= 1 && pmax >= k - 1) {
                    // every split point 1..k-1: the loads of split s + 1 are
                    // issued before the FMAs of split s
                    T lv[D];
                    TR rv[V];
                    auto load = [&](int sd) {
                        const int p = k - sd;
                        const T* lp = lhs + a.db[p] + q;
                        const uint32_t dp1 = (uint32_t)a.pw[p - 1];
#pragma unroll
                        for (int u = 0; u < D; ++u) lv[u] = __ldg(lp + u * dp1);
                        const TR* rq = rhs + a.db[sd] + (int64_t)m * D + c0;
#pragma unroll
                        for (int j = 0; j < V; ++j) rv[j] = __ldg(rq + j);
                    };
                    auto peel = [&](int sd) {
                        const uint32_t q2 = q / (uint32_t)D;
                        m += (q - q2 * (uint32_t)D) * (uint32_t)a.pw[sd - 1];
                        q = q2;
                    };
                    if (k >= 2) load(1);
                    for (int sd = 1; sd <= k - 1; ++sd) {
                        T cl[D];
                        TR cr[V];
#pragma unroll
                        for (int u = 0; u < D; ++u) cl[u] = lv[u];
#pragma unroll
                        for (int j = 0; j < V; ++j) cr[j] = rv[j];
                        peel(sd);
                        if (sd + 1 <= k - 1) load(sd + 1);
#pragma unroll
                        for (int u = 0; u < D; ++u)
#pragma unroll
                            for (int j = 0; j < V; ++j) acc[u][j].add(cl[u], T(cr[j]));
                    }
                } else {
                    for (int s = 1; s <= k - 1; ++s) {
                        const int p = k - s;
                        if (p <= pmax && p >= pmin) {
                            T lv[D];
                            T rv[V];
                            const T* lp = lhs + a.db[p] + q;
                            const uint32_t dp1 = (uint32_t)a.pw[p - 1];
#pragma unroll
                            for (int u = 0; u < D; ++u) lv[u] = __ldg(lp + u * dp1);
                            const TR* rq = rhs + a.db[s] + (int64_t)m * D + c0;
#pragma unroll
                            for (int j = 0; j < V; ++j) rv[j] = T(__ldg(rq + j));
#pragma unroll
                            for (int u = 0; u < D; ++u)
#pragma unroll
                                for (int j = 0; j < V; ++j) acc[u][j].add(lv[u], rv[j]);
                        }
                        const uint32_t q2 = q / (uint32_t)D;
                        m += (q - q2 * (uint32_t)D) * (uint32_t)a.pw[s - 1];
                        q = q2;
                    }
                }
                if (pmin <= 0 && pmax >= 0) {
                    const TR* rk = rhs + obase;
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j)
                            acc[u][j].add(lhs0, T(__ldg(rk + u * dk1 + j)));
                }
            }

            const T sc = T(a.scale[k]);
#pragma unroll
            for (int u = 0; u < D; ++u)
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const int64_t o = obase + u * dk1 + j;
                    T v;
                    if (a.accumulate) {
                        v = acc[u][j].value();
                    } else {
                        v = sc * acc[u][j].value();
                        if (add) v += add[o];
                    }
                    out[o] = v;
                }
        }
    }
}

// Blocked variant owning the last L >= 2 letters (V = D^L combinations): a
// thread computes the D x V words u d^(k-1) + r' V + j for one middle part
// r' (k-1-L letters), for output levels k > L.  Split points with a right
// part of s >= L letters share D left words and V right words as above;
// the s < L splits cut into the owned letters and load D d^(L-s) left and
// d^s right words.
template <typename T, typename TR, int D, int L, int ACC = 0, int MINB = 1>
__global__ void __launch_bounds__(kThreads, MINB)
product_kernel_blocked_l(const KArgs a)
{
    constexpr int V = (L == 2) ? D * D : D * D * D;
    using AccT = typename AccSel<T, ACC>::type;
    const int64_t f_begin = (int64_t)blockIdx.x * a.tile_r;
    const int64_t f_end = min(f_begin + a.tile_r, a.ftotal);

    for (int64_t b = blockIdx.y; b < a.batch; b += gridDim.y) {
        const int64_t ro = a.out_idx ? a.out_idx[b] : b;
        const int64_t rl = a.lhs_idx ? a.lhs_idx[b] : b;
        const int64_t rr = a.rhs_idx ? a.rhs_idx[b] : b;
        T* __restrict__ out = static_cast<T*>(a.out) + ro * a.ld_out;
        const T* __restrict__ lhs = static_cast<const T*>(a.lhs) + rl * a.ld_lhs;
        const TR* __restrict__ rhs = static_cast<const TR*>(a.rhs) + rr * a.ld_rhs;
        const T* __restrict__ add =
            a.addend ? static_cast<const T*>(a.addend) + ro * a.ld_add : nullptr;
        const T lhs0 = (a.lhs0_from_mem ? __ldg(lhs) : T(0)) + T(a.lhs0_add);
        const T rhs0 = T(__ldg(rhs));
        if (blockIdx.x == 0) small_levels<T, TR, AccT>(a, out, lhs, rhs, add, lhs0);

        for (int64_t f = f_begin + threadIdx.x; f < f_end; f += kThreads) {
            int k = a.klo;
            while (f >= a.fcum[k + 1]) ++k;
            const uint32_t rp = (uint32_t)(f - a.fcum[k]);
            const int64_t dk1 = a.pw[k - 1];
            const int64_t obase = a.db[k] + (int64_t)rp * V;
            if (a.prefetch && a.pmin[k] <= 0 && a.pmax[k] >= 0) {
#pragma unroll
                for (int u = 0; u < D; ++u) prefetch_l2(rhs + obase + u * dk1);
            }

            AccT acc[D][V];
#pragma unroll
            for (int u = 0; u < D; ++u)
#pragma unroll
                for (int j = 0; j < V; ++j)
                    acc[u][j].init(a.accumulate ? out[obase + u * dk1 + j] : T(0));

            const int pmax = a.pmax[k];
            const int pmin = a.pmin[k];
            if (pmax >= pmin) {
                if (k <= pmax && k >= pmin) {
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j)
                            acc[u][j].add(__ldg(lhs + obase + u * dk1 + j), rhs0);
                }
                // splits cutting into the owned letters: right part j mod D^s
#pragma unroll
                for (int s = 1; s < L; ++s) {
                    const int p = k - s;
                    if (p <= pmax && p >= pmin) {
                        constexpr int dummy = 0;
                        (void)dummy;
                        const int ds = (s == 1) ? D : D * D;          // D^s (L <= 3)
                        const int dl = V / ds;                          // D^(L-s)
                        const uint32_t dp1 = (uint32_t)a.pw[p - 1];
                        const T* lp = lhs + a.db[p] + (int64_t)rp * dl;
                        const TR* rq = rhs + a.db[s];
#pragma unroll
                        for (int u = 0; u < D; ++u)
#pragma unroll
                            for (int j = 0; j < V; ++j)
                                acc[u][j].add(__ldg(lp + u * dp1 + j / ds), T(__ldg(rq + j % ds)));
                    }
                }
                // splits with a right part of s >= L letters
                uint32_t q = rp;
                uint32_t m = 0;
                for (int s = L; s <= k - 1; ++s) {
                    const int p = k - s;
                    if (p <= pmax && p >= pmin) {
                        T lv[D];
                        T rv[V];
                        const T* lp = lhs + a.db[p] + q;
                        const uint32_t dp1 = (uint32_t)a.pw[p - 1];
#pragma unroll
                        for (int u = 0; u < D; ++u) lv[u] = __ldg(lp + u * dp1);
                        const TR* rq = rhs + a.db[s] + (int64_t)m * V;
#pragma unroll
                        for (int j = 0; j < V; ++j) rv[j] = T(__ldg(rq + j));
#pragma unroll
                        for (int u = 0; u < D; ++u)
#pragma unroll
                            for (int j = 0; j < V; ++j) acc[u][j].add(lv[u], rv[j]);
                    }
                    const uint32_t q2 = q / (uint32_t)D;
                    m += (q - q2 * (uint32_t)D) * (uint32_t)a.pw[s - L];
                    q = q2;
                }
                if (pmin <= 0 && pmax >= 0) {
                    const TR* rk = rhs + obase;
#pragma unroll
                    for (int u = 0; u < D; ++u)
#pragma unroll
                        for (int j = 0; j < V; ++j)
                            acc[u][j].add(lhs0, T(__ldg(rk + u * dk1 + j)));
                }
            }

            const T sc = T(a.scale[k]);
#pragma unroll
            for (int u = 0; u < D; ++u)
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const int64_t o = obase + u * dk1 + j;
                    T v;
                    if (a.accumulate) {
                        v = acc[u][j].value();
                    } else {
                        v = sc * acc[u][j].value();
                        if (add) v += add[o];
                    }
                    out[o] = v;
                }
        }
    }
}

// Width-2 kernel for output levels k >= 6 + E (H = 2^E): the 32 lanes of a
// warp own the last five letters of a word, so that every right-factor run
// and every streamed top-level word is one coalesced request and every
// left-factor word one broadcast.  (The blocked kernels above give a thread
// V consecutive words, and their loads of one word per thread are 32 bytes
// apart across the warp.)  A thread owns the 2 H words
//   w(u, i) = u 2^(k-1) + (h0 + i) 32 + lane      (u < 2, i < H)
// for one block h0 (a multiple of H) of middle parts.  A split point with a
// right part of s letters (left part p = k - s) reads
//   s >= 5 + E:      L_p[u 2^(p-1) + (h0 >> (s-5))] (2 broadcasts) and the
//                    H runs R_s[((h0 mod 2^(s-5)) + i) 32 + lane];
//   5 <= s < 5 + E:  L_p[u 2^(p-1) + (h0 >> e) + (i >> e)] and
//                    R_s[(i mod 2^e) 32 + lane], e = s - 5;
//   s < 5:           R_s[lane mod 2^s] (one word per lane) and the 2 H runs
//                    L_p[u 2^(p-1) + (h0 + i) 2^(5-s) + (lane >> s)].
// The terms of a word are added in the same order as in the other kernels
// (left degree from k down to 0), so the results are the same bits.  Index
// arithmetic is 32-bit within a row; level k starts at word 2^k - 1.
template <typename T, typename TR, int H, int ACC = 0, int MINB = 1>
__global__ void __launch_bounds__(kThreads, MINB)
product_kernel_w2(const KArgs a)
{
    constexpr int E = (H == 1) ? 0 : (H == 2) ? 1 : (H == 4) ? 2 : 3;
    static_assert((1 << E) == H, "H must be 1, 2, 4 or 8");
    using AccT = typename AccSel<T, ACC>::type;
    const int64_t f_begin = (int64_t)blockIdx.x * a.tile_r;
    const int64_t f_end = min(f_begin + a.tile_r, a.ftotal);
    const uint32_t lane = threadIdx.x & 31u;

    for (int64_t b = blockIdx.y; b < a.batch; b += gridDim.y) {
        const int64_t ro = a.out_idx ? a.out_idx[b] : b;
        const int64_t rl = a.lhs_idx ? a.lhs_idx[b] : b;
        const int64_t rr = a.rhs_idx ? a.rhs_idx[b] : b;
        T* __restrict__ out = static_cast<T*>(a.out) + ro * a.ld_out;
        const T* __restrict__ lhs = static_cast<const T*>(a.lhs) + rl * a.ld_lhs;
        const TR* __restrict__ rhs = static_cast<const TR*>(a.rhs) + rr * a.ld_rhs;
        const T* __restrict__ add =
            a.addend ? static_cast<const T*>(a.addend) + ro * a.ld_add : nullptr;
        const T lhs0 = (a.lhs0_from_mem ? __ldg(lhs) : T(0)) + T(a.lhs0_add);
        const T rhs0 = T(__ldg(rhs));
        if (blockIdx.x == 0) small_levels<T, TR, AccT, true>(a, out, lhs, rhs, add, lhs0);

        // a warp's 32 consecutive units share k and h0 (tiles and level
        // starts are multiples of 32 units)
        for (int64_t f = f_begin + threadIdx.x; f < f_end; f += kThreads) {
            int k = a.klo;
            while (f >= a.fcum[k + 1]) ++k;
            const uint32_t rp = (uint32_t)(f - a.fcum[k]);
            const uint32_t h0 = (rp >> 5) << E;
            const uint32_t half = 1u << (k - 1);
            const uint32_t wb = ((1u << k) - 1u) + h0 * 32u + lane;   // word (0, 0) in the row
            if (a.prefetch && a.pmin[k] <= 0 && a.pmax[k] >= 0) {
#pragma unroll
                for (int u = 0; u < 2; ++u)
#pragma unroll
                    for (int i = 0; i < H; ++i) prefetch_l2(rhs + wb + u * half + 32u * i);
            }

            AccT acc[2][H];
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int i = 0; i < H; ++i)
                    acc[u][i].init(a.accumulate ? out[wb + u * half + 32u * i] : T(0));

            const int pmax = a.pmax[k];
            const int pmin = a.pmin[k];
            if (pmax >= pmin) {
                if (k <= pmax && k >= pmin) {
#pragma unroll
                    for (int u = 0; u < 2; ++u)
#pragma unroll
                        for (int i = 0; i < H; ++i)
                            acc[u][i].add(__ldg(lhs + wb + u * half + 32u * i), rhs0);
                }
                // right parts of 1..4 letters: one right word per lane
#pragma unroll
                for (int s = 1; s <= 4; ++s) {
                    const int p = k - s;
                    if (p <= pmax && p >= pmin) {
                        const T rv = T(__ldg(rhs + ((1u << s) - 1u) + (lane & ((1u << s) - 1u))));
                        const uint32_t lb = ((1u << p) - 1u) + h0 * (32u >> s) + (lane >> s);
                        const uint32_t lh = 1u << (p - 1);
#pragma unroll
                        for (int u = 0; u < 2; ++u)
#pragma unroll
                            for (int i = 0; i < H; ++i)
                                acc[u][i].add(__ldg(lhs + lb + u * lh + (32u >> s) * i), rv);
                    }
                }
                // right parts of 5 .. 4 + E letters
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int s = 5 + e;
                    const int p = k - s;
                    if (p <= pmax && p >= pmin) {
                        const int nr = 1 << e;
                        T rv[H];
#pragma unroll
                        for (int c = 0; c < nr; ++c)
                            rv[c] = T(__ldg(rhs + ((1u << s) - 1u) + 32u * c + lane));
                        const uint32_t lb = ((1u << p) - 1u) + (h0 >> e);
                        const uint32_t lh = 1u << (p - 1);
#pragma unroll
                        for (int u = 0; u < 2; ++u)
#pragma unroll
                            for (int g = 0; g < (H >> e); ++g) {
                                const T lv = __ldg(lhs + lb + u * lh + g);
#pragma unroll
                                for (int c = 0; c < nr; ++c) acc[u][g * nr + c].add(lv, rv[c]);
                            }
                    }
                }
                // right parts of 5 + E .. k - 1 letters: H runs, 2 broadcasts
                for (int s = 5 + E; s <= k - 1; ++s) {
                    const int p = k - s;
                    if (p <= pmax && p >= pmin) {
                        const uint32_t rb =
                            ((1u << s) - 1u) + (h0 & ((1u << (s - 5)) - 1u)) * 32u + lane;
                        T rv[H];
#pragma unroll
                        for (int i = 0; i < H; ++i) rv[i] = T(__ldg(rhs + rb + 32u * i));
                        const uint32_t lb = ((1u << p) - 1u) + (h0 >> (s - 5));
                        const T lv0 = __ldg(lhs + lb);
                        const T lv1 = __ldg(lhs + lb + (1u << (p - 1)));
#pragma unroll
                        for (int i = 0; i < H; ++i) {
                            acc[0][i].add(lv0, rv[i]);
                            acc[1][i].add(lv1, rv[i]);
                        }
                    }
                }
                if (pmin <= 0 && pmax >= 0) {
#pragma unroll
                    for (int u = 0; u < 2; ++u)
#pragma unroll
                        for (int i = 0; i < H; ++i)
                            acc[u][i].add(lhs0, T(__ldg(rhs + wb + u * half + 32u * i)));
                }
            }

            const T sc = T(a.scale[k]);
#pragma unroll
            for (int u = 0; u < 2; ++u)
#pragma unroll
                for (int i = 0; i < H; ++i) {
                    const uint32_t o = wb + u * half + 32u * i;
                    T v;
                    if (a.accumulate) {
                        v = acc[u][i].value();
                    } else {
                        v = sc * acc[u][i].value();
                        if (add) v += add[o];
                    }
                    out[o] = v;
                }
        }
    }
}

template <typename TD, typename TS>
__global__ void convert_rows_kernel(TD* dst, int64_t ld_dst, const TS* src, int64_t ld_src,
                                    int64_t cols, int64_t batch)
{
    const int64_t total = cols * batch;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = i / cols;
        const int64_t c = i - b * cols;
        dst[b * ld_dst + c] = static_cast<TD>(src[b * ld_src + c]);
    }
}

template <typename T, typename TR, int ACC>
int dispatch(const KArgs& a, dim3 grid, cudaStream_t stream)
{
    switch (a.width) {
        case 2: product_kernel<T, TR, 2, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        case 3: product_kernel<T, TR, 3, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        case 4: product_kernel<T, TR, 4, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        case 5: product_kernel<T, TR, 5, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        case 6: product_kernel<T, TR, 6, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        case 7: product_kernel<T, TR, 7, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        case 8: product_kernel<T, TR, 8, ACC><<<grid, kThreads, 0, stream>>>(a); break;
        default:
            if (a.width > 16) return fail(RPYB_E_UNSUPPORTED, "product kernel supports width <= 16");
            product_kernel<T, TR, 0, ACC><<<grid, kThreads, 0, stream>>>(a);
            break;
    }
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

int f32_acc_mode()
{
    static int m = [] {
        const char* e = getenv("RPYB_F32_ACC");
        if (!e) return 1;            // float64 accumulation
        if (e[0] == 'd') return 0;   // "df": double-float pair
        if (e[0] == 'p') return 2;   // "plain"
        return 1;
    }();
    return m;
}

int tile_words()
{
    static int w = [] {
        const char* e = getenv("RPYB_TILE_WORDS");
        int v = e ? atoi(e) : 4096;
        return v >= 256 ? v : 4096;
    }();
    return w;
}

// float32 rows at width 8 own four last letters per thread (twice the
// float64 block), so each thread keeps as many bytes in flight as a float64
// one (measured on B200: (8,6) 1.36 -> 1.27 ms; a block of six at width 6
// was slower, so width 6 keeps three).  RPYB_F32_WIDE=0 restores two.
// RPYB_PRODUCT_PREFETCH=0: no L2 prefetch of the streamed right words
// (measured on B200, batch 1024: +3 to +8 % of HBM at (4,8) and (6,6))
bool product_prefetch()
{
    static const bool on = [] {
        const char* e = getenv("RPYB_PRODUCT_PREFETCH");
        return !(e && e[0] == '0');
    }();
    return on;
}

// RPYB_PRODUCT_PIPE=0: the width-8 float32 blocked kernel walks its split
// points without software pipelining
bool product_pipe()
{
    static const bool on = [] {
        const char* e = getenv("RPYB_PRODUCT_PIPE");
        return !(e && e[0] == '0');
    }();
    return on;
}

bool f32_wide_blocks()
{
    static const bool on = [] {
        const char* e = getenv("RPYB_F32_WIDE");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Width -> last-letter block V of the one-letter blocked kernel (0: none);
// float64 rows at width 4 use a block of 2 (more resident warps)
int blocked_v_one(int width, bool f64 = false)
{
    switch (width) {
        case 3: return 3;
        case 4: return f64 ? 2 : 4;
        case 5: return 5;
        case 6: return 3;
        case 8: return (!f64 && f32_wide_blocks()) ? 4 : 2;
        default: return 0;
    }
}

// Width 2 owns its last 2 letters (RPYB_W2_LETTERS=3: three; two measured
// faster on B200)
int width2_letters()
{
    static const int l = [] {
        const char* e = getenv("RPYB_W2_LETTERS");
        return (e && e[0] == '3') ? 3 : 2;
    }();
    return l;
}

// Width -> number of owned last letters of the blocked kernels (0: none)
int blocked_l(int width)
{
    if (width == 2) return width2_letters();
    return blocked_v_one(width) ? 1 : 0;
}

// Width -> owned last-letter combinations V per thread
int blocked_v(int width, bool f64)
{
    if (width == 2) return width2_letters() == 2 ? 4 : 8;
    return blocked_v_one(width, f64);
}

// RPYB_PRODUCT_BLOCKED=0 keeps every level on the suffix kernel
bool blocked_enabled()
{
    static const bool on = [] {
        const char* e = getenv("RPYB_PRODUCT_BLOCKED");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename T, typename TR, int ACC>
int dispatch_blocked(const KArgs& a, dim3 grid, cudaStream_t stream)
{
    if (a.width == 2) {
        if (width2_letters() == 2)
            product_kernel_blocked_l<T, TR, 2, 2, ACC, 5><<<grid, kThreads, 0, stream>>>(a);
        else
            product_kernel_blocked_l<T, TR, 2, 3, ACC, 3><<<grid, kThreads, 0, stream>>>(a);
        RPYB_CUDA(cudaGetLastError());
        return RPYB_OK;
    }
    // the pipelined split loop for float32 rows at width 8 (float64
    // accumulation); measured on B200, % of HBM: (8,6) 62.8 -> 65.2,
    // (8,5) 61.4 -> 65.7, but width 6 61.5 -> 60.6, so width 6 keeps the plain loop
    const bool pipe = product_pipe() && sizeof(T) == 4 && ACC == 1;
    switch (a.width) {
        // last-letter blocks and resident blocks per SM (register caps) from
        // measurements on B200
        case 3: product_kernel_blocked<T, TR, 3, 3, ACC, 4><<<grid, kThreads, 0, stream>>>(a); break;
        case 4:
            if (sizeof(T) == 8)
                product_kernel_blocked<T, TR, 4, 2, ACC, 4><<<grid, kThreads, 0, stream>>>(a);
            else
                product_kernel_blocked<T, TR, 4, 4, ACC, 4><<<grid, kThreads, 0, stream>>>(a);
            break;
        case 5: product_kernel_blocked<T, TR, 5, 5, ACC, 2><<<grid, kThreads, 0, stream>>>(a); break;
        case 6:
            // float32 rows: four resident blocks (a few spilled registers cost
            // less than the lost occupancy)
            if (sizeof(T) == 4)
                product_kernel_blocked<T, TR, 6, 3, ACC, 4><<<grid, kThreads, 0, stream>>>(a);
            else
                product_kernel_blocked<T, TR, 6, 3, ACC, 3><<<grid, kThreads, 0, stream>>>(a);
            break;
        case 8:
            if (sizeof(T) == 4 && sizeof(TR) == 4 && f32_wide_blocks()) {
                if (pipe)
                    product_kernel_blocked<T, TR, 8, 4, ACC, 2, true><<<grid, kThreads, 0, stream>>>(a);
                else
                    product_kernel_blocked<T, TR, 8, 4, ACC, 2><<<grid, kThreads, 0, stream>>>(a);
            } else {
                product_kernel_blocked<T, TR, 8, 2, ACC, 3><<<grid, kThreads, 0, stream>>>(a);
            }
            break;
        default: return fail(RPYB_E_UNSUPPORTED, "no blocked product kernel for this width");
    }
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

// Width 2 from level kW2Low up, float64 rows: product_kernel_w2 with H =
// kW2H middle parts per thread (RPYB_W2_KERNEL=0 keeps the blocked kernel).
// Measured on B200, config 2 at (2,12), % of HBM: float64 46 -> 61; float32
// rows 35 -> 33 (their F2F conversions bound them, and this kernel converts
// every loaded word), so float32 and mixed rows keep the blocked kernel.
constexpr int kW2H = 4;
constexpr int kW2Low = 8;   // 6 + log2(kW2H): 2^(k-1) >= 32 kW2H words per first letter
// products whose top level is at least this take the kernel.  Below it the
// levels under kW2Low, computed word by word in one tile per row, weigh too
// much: config-2 sweep on B200, float64 % of HBM, lane-letter / blocked:
// depth 12 61 / 46, 11 50 / 43, 10 37 / 35, 9 22 / 24, 8 11 / 13
constexpr int kW2MinTop = 10;

bool w2_kernel_enabled()
{
    static const bool on = [] {
        const char* e = getenv("RPYB_W2_KERNEL");
        return !(e && e[0] == '0');
    }();
    return on;
}

// five resident blocks (48 registers); four were slower on B200 ((2,12):
// 53 against 61 % of HBM)
int dispatch_w2(const KArgs& a, dim3 grid, cudaStream_t stream)
{
    product_kernel_w2<double, double, kW2H, 0, 5><<<grid, kThreads, 0, stream>>>(a);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

}  // namespace

enum LaunchMode { kSuffix = 0, kBlocked = 1, kW2 = 2 };

static int launch_levels(int dtype, const Geometry& g, const ProductSpec& spec,
                         const ProductRows& rows, cudaStream_t stream, int mode);

int launch_product(int dtype, const Geometry& g, const ProductSpec& spec,
                   const ProductRows& rows, cudaStream_t stream)
{
    if (rows.batch <= 0) return RPYB_OK;
    // float64 rows of width 2 up to level kW2MinTop or higher: the
    // lane-letter kernel
    if (dtype == RPYB_F64 && blocked_enabled() && g.width == 2 && w2_kernel_enabled() &&
        spec.khi >= kW2MinTop)
        return launch_levels(dtype, g, spec, rows, stream, kW2);
    const int L = blocked_enabled() ? blocked_l(g.width) : 0;
    const int kb = std::max(L + 1, spec.klo);
    if (L == 0 || spec.khi < kb) return launch_levels(dtype, g, spec, rows, stream, kSuffix);
    // one blocked launch: levels kb..khi by units, levels klo..L and the
    // level-0 rule word by word in each row's first tile
    return launch_levels(dtype, g, spec, rows, stream, kBlocked);
}

static int launch_levels(int dtype, const Geometry& g, const ProductSpec& spec,
                         const ProductRows& rows, cudaStream_t stream, int mode)
{
    const bool blocked = mode != kSuffix;
    KArgs a{};
    a.width = g.width;
    a.klo = std::max(1, spec.klo);
    a.khi = spec.khi;
    a.sklo = 1;
    a.skhi = 0;
    if (blocked) {
        const int Lb = mode == kW2 ? kW2Low - 1 : blocked_l(g.width);
        a.sklo = a.klo;
        a.skhi = std::min(spec.khi, Lb);
        a.klo = std::max(Lb + 1, spec.klo);
    }
    for (int i = 0; i <= kMaxDepth + 1; ++i) a.db[i] = g.db[i];
    for (int i = 0; i <= kMaxDepth; ++i) a.pw[i] = g.pw[i];
    int64_t f = 0;
    for (int k = 0; k <= kMaxDepth + 1; ++k) a.fcum[k] = 0;
    // work units per level: suffixes (one per d^(k-1)) or, blocked, one per
    // middle part and last-letter block (d^(k-2) * d / V)
    const int V = mode == kW2 ? 2 * kW2H : blocked ? blocked_v(g.width, dtype != RPYB_F32) : 0;
    const int L = mode == kBlocked ? blocked_l(g.width) : 0;
    for (int k = a.klo; k <= a.khi; ++k) {
        a.fcum[k] = f;
        if (mode == kW2) f += g.pw[k - 1] / kW2H;   // a multiple of 32 for k >= kW2Low
        else if (!blocked) f += g.pw[k - 1];
        else if (L == 1) f += g.pw[k - 2] * (g.width / V);
        else f += g.pw[k - 1 - L];
    }
    // sentinel entries above khi so the level search stops
    for (int k = std::max(a.khi + 1, a.klo); k <= kMaxDepth + 1; ++k) a.fcum[k] = f;
    a.ftotal = f;
    for (int k = 0; k <= kMaxDepth; ++k) {
        a.pmin[k] = spec.pmin[k];
        a.pmax[k] = spec.pmax[k];
        a.scale[k] = spec.scale[k];
    }
    a.accumulate = spec.accumulate;
    a.lhs0_from_mem = spec.lhs0_from_mem;
    a.lhs0_add = spec.lhs0_add;
    a.l0_write = spec.l0_write;
    a.l0_prod = spec.l0_prod;
    a.l0_base = spec.l0_base;
    a.l0_const = spec.l0_const;
    a.scale0 = spec.scale0;
    a.out = rows.out;
    a.lhs = rows.lhs;
    a.rhs = rows.rhs;
    a.addend = rows.addend;
    a.ld_out = rows.ld_out;
    a.ld_lhs = rows.ld_lhs;
    a.ld_rhs = rows.ld_rhs;
    a.ld_add = rows.ld_add;
    a.out_idx = rows.out_idx;
    a.lhs_idx = rows.lhs_idx;
    a.rhs_idx = rows.rhs_idx;
    a.batch = rows.batch;
    a.prefetch = blocked && product_prefetch();

    // Work units per tile: about kTileWords output words per CTA (at least
    // one unit per thread).
    const int64_t words_per_unit = mode == kW2 ? V : blocked ? (int64_t)g.width * V : g.width;
    a.tile_r = std::max<int64_t>(kThreads, tile_words() / std::max<int64_t>(1, words_per_unit));
    int64_t tiles = (a.ftotal + a.tile_r - 1) / a.tile_r;
    if (tiles == 0) tiles = 1;  // level 0 only
    if (tiles > 0x7fffffff) return fail(RPYB_E_UNSUPPORTED, "tensor too large");
    dim3 grid((unsigned)tiles, (unsigned)std::min<int64_t>(rows.batch, 65535), 1);
    if (mode == kW2) return dispatch_w2(a, grid, stream);   // float64 rows only
    if (blocked) {
        if (dtype == RPYB_F64) return dispatch_blocked<double, double, 0>(a, grid, stream);
        if (dtype == kMixedF64F32) return dispatch_blocked<double, float, 0>(a, grid, stream);
        switch (f32_acc_mode()) {
            case 1: return dispatch_blocked<float, float, 1>(a, grid, stream);
            case 2: return dispatch_blocked<float, float, 2>(a, grid, stream);
            default: return dispatch_blocked<float, float, 0>(a, grid, stream);
        }
    }
    if (dtype == RPYB_F64) return dispatch<double, double, 0>(a, grid, stream);
    if (dtype == kMixedF64F32) return dispatch<double, float, 0>(a, grid, stream);
    switch (f32_acc_mode()) {
        case 1: return dispatch<float, float, 1>(a, grid, stream);
        case 2: return dispatch<float, float, 2>(a, grid, stream);
        default: return dispatch<float, float, 0>(a, grid, stream);
    }
}

int launch_convert_rows(int dst_dtype, void* dst, int64_t ld_dst, int src_dtype,
                        const void* src, int64_t ld_src, int64_t cols, int64_t batch,
                        cudaStream_t stream)
{
    if (cols <= 0 || batch <= 0) return RPYB_OK;
    const int64_t total = cols * batch;
    const int threads = 256;
    const int64_t blocks = std::min<int64_t>((total + threads - 1) / threads, 148 * 32);
    if (dst_dtype == RPYB_F64 && src_dtype == RPYB_F32) {
        convert_rows_kernel<double, float><<<(unsigned)blocks, threads, 0, stream>>>(
            static_cast<double*>(dst), ld_dst, static_cast<const float*>(src), ld_src, cols, batch);
    } else if (dst_dtype == RPYB_F32 && src_dtype == RPYB_F64) {
        convert_rows_kernel<float, double><<<(unsigned)blocks, threads, 0, stream>>>(
            static_cast<float*>(dst), ld_dst, static_cast<const double*>(src), ld_src, cols, batch);
    } else if (dst_dtype == RPYB_F64) {
        convert_rows_kernel<double, double><<<(unsigned)blocks, threads, 0, stream>>>(
            static_cast<double*>(dst), ld_dst, static_cast<const double*>(src), ld_src, cols, batch);
    } else {
        convert_rows_kernel<float, float><<<(unsigned)blocks, threads, 0, stream>>>(
            static_cast<float*>(dst), ld_dst, static_cast<const float*>(src), ld_src, cols, batch);
    }
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

}  // namespace rpyb
