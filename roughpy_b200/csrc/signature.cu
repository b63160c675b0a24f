// Batched path signatures on sm_100a: S = exp(x_0) (x) exp(x_1) (x) ... for
// thousands of streams of uneven length in one persistent launch.
//
// Decomposition.  For a level-1 increment x the Chen step S <- S (x) exp(x)
// updates word w = (a_1 .. a_k) from S restricted to the prefixes of w:
//
//   S'_k[w] = sum_{j=0..k} S_{k-j}[a_1..a_{k-j}] x[a_{k-j+1}] ... x[a_k] / j!
//
// so the words under a fixed prefix evolve independently of every other
// subtree.  One lane owns a level-(N-2) word pi (its "path" is the prefix
// chain pi_1, pi_1 pi_2, ..., pi), G of pi's children at level N-1 and the
// G*D top words below them.  The lane keeps everything it needs in
// registers and recomputes the few shared ancestors (levels <= N-2) itself,
// so lanes never communicate: there is no __syncthreads and no shared
// state.  A warp takes 32 consecutive lanes of one stream from a device-side
// queue (longest streams first) and walks that stream's increments.
//
// Per step, level k is evaluated by the Horner chain
//   acc_1 = S_1 + x/k,  acc_i = S_i + acc_{i-1} (x) x/(k-i+1),  S'_k = S_k + acc_{k-1} (x) x
// restricted to the lane's words, processing levels from the top down so that
// every chain reads pre-step values (free_tensor_inplace_mul.hpp:22-85 uses the
// same top-down order).
//
// Precision modes.  float64: plain double state and FMAs.  float32
// ("compensated"): the products are float32, each word keeps its running
// value as hi + lo plus a float32 delta accumulator that receives the step's
// increment with one FMA (top-level words two at a time with packed f32x2
// FMAs); every `fold` steps (default 24) the delta is folded into (hi, lo)
// with an exact two-sum and (hi, lo) is renormalised so that hi is the
// rounded value.  Chains read hi + delta.  The top level's lo words (and at
// width 8 its hi words too) live in shared memory: they are touched only
// when folding, which leaves the registers to the delta accumulators.
#include <algorithm>
#include <initializer_list>
#include <mutex>
#include <tuple>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "signature_internal.cuh"

namespace rpyb {
namespace {

constexpr int kSigWarps = 8;  // warps per block of the persistent kernel
constexpr int kChunk = 32;    // increment rows staged per warp in shared memory

// register cap of the float32 split kernel: without it the compiler hoists
// the fold's shared-memory loads and uses over 230 registers at width 8;
// 192 fits ten warps per SM (the shared-memory limit at width 8) unspilled
#ifndef RPYB_SIG_SPLIT_MAXREG
#define RPYB_SIG_SPLIT_MAXREG 192
#endif
// with the top level in TMEM shared memory no longer limits the warps per
// SM; 168 registers fit three blocks of four warps
#ifndef RPYB_SIG_TMEM_MAXREG
#define RPYB_SIG_TMEM_MAXREG 168
#endif

// level-(N-1) words per lane of the float64 kernel at width 8
#ifndef RPYB_SIG_F64_G8
#define RPYB_SIG_F64_G8 8
#endif

struct SigArgs {
    const int64_t* offsets;
    const void* inc;
    void* out;
    int64_t ld_out;
    const int64_t* order;
    int64_t n_streams;
    int64_t items_per_stream;
    int64_t total_items;
    int* queue;   // device work counter (zeroed before launch)
    int fold;     // fold interval of the classic compensated mode (steps)
    int fold_chunks;  // split kernel: chunks of kChunk steps between folds
    // output rows: row s of `out` unless dst_row is given, in which case
    // r = dst_row[s] selects row r of `out` (r >= 0) or row ~r of `alt`
    // (r < 0; the segment rows of split streams)
    const int64_t* dst_row;
    void* alt;
    int64_t ld_alt;
    int64_t db[kMaxDepth + 2];
};

template <typename T>
__device__ __forceinline__ T* output_row(const SigArgs& a, int64_t s)
{
    if (a.dst_row == nullptr) return static_cast<T*>(a.out) + s * a.ld_out;
    const int64_t r = a.dst_row[s];
    return r >= 0 ? static_cast<T*>(a.out) + r * a.ld_out : static_cast<T*>(a.alt) + (~r) * a.ld_alt;
}

template <int D, int E>
struct IPow {
    static constexpr int64_t value = D * IPow<D, E - 1>::value;
};
template <int D>
struct IPow<D, 0> {
    static constexpr int64_t value = 1;
};

template <typename T, int D>
__device__ __forceinline__ void load_row(T (&x)[D], const T* __restrict__ p)
{
    if constexpr (sizeof(T) == 4 && (D % 4) == 0) {
#pragma unroll
        for (int i = 0; i < D / 4; ++i) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p) + i);
            x[4 * i + 0] = v.x;
            x[4 * i + 1] = v.y;
            x[4 * i + 2] = v.z;
            x[4 * i + 3] = v.w;
        }
    } else if constexpr (sizeof(T) == 8 && (D % 2) == 0) {
#pragma unroll
        for (int i = 0; i < D / 2; ++i) {
            const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
            x[2 * i + 0] = v.x;
            x[2 * i + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < D; ++i) x[i] = __ldg(p + i);
    }
}

template <typename T, int D>
__device__ __forceinline__ void store_row(T* __restrict__ p, const T (&x)[D])
{
    if constexpr (sizeof(T) == 4 && (D % 4) == 0) {
#pragma unroll
        for (int i = 0; i < D / 4; ++i)
            reinterpret_cast<float4*>(p)[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2],
                                                          x[4 * i + 3]);
    } else if constexpr (sizeof(T) == 8 && (D % 2) == 0) {
#pragma unroll
        for (int i = 0; i < D / 2; ++i)
            reinterpret_cast<double2*>(p)[i] = make_double2(x[2 * i], x[2 * i + 1]);
    } else {
#pragma unroll
        for (int i = 0; i < D; ++i) p[i] = x[i];
    }
}

template <typename T, int D>
__device__ __forceinline__ void load_row_smem(T (&x)[D], const T* __restrict__ p)
{
    if constexpr (sizeof(T) == 4 && (D % 4) == 0) {
#pragma unroll
        for (int i = 0; i < D / 4; ++i) {
            const float4 v = reinterpret_cast<const float4*>(p)[i];
            x[4 * i + 0] = v.x;
            x[4 * i + 1] = v.y;
            x[4 * i + 2] = v.z;
            x[4 * i + 3] = v.w;
        }
    } else if constexpr (sizeof(T) == 8 && (D % 2) == 0) {
#pragma unroll
        for (int i = 0; i < D / 2; ++i) {
            const double2 v = reinterpret_cast<const double2*>(p)[i];
            x[2 * i + 0] = v.x;
            x[2 * i + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < D; ++i) x[i] = p[i];
    }
}

template <typename T, int K>
__device__ __forceinline__ void load_slice(T (&v)[K], const T* __restrict__ p)
{
    // vector loads when the slice is a whole number of 16-byte chunks and
    // starts on a 16-byte boundary (true for the shapes that use them)
    if constexpr ((K * sizeof(T)) % 16 == 0) {
        if constexpr (sizeof(T) == 4) {
#pragma unroll
            for (int i = 0; i < K / 4; ++i) {
                const float4 q = reinterpret_cast<const float4*>(p)[i];
                v[4 * i] = q.x;
                v[4 * i + 1] = q.y;
                v[4 * i + 2] = q.z;
                v[4 * i + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int i = 0; i < K / 2; ++i) {
                const double2 q = reinterpret_cast<const double2*>(p)[i];
                v[2 * i] = q.x;
                v[2 * i + 1] = q.y;
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < K; ++i) v[i] = p[i];
    }
}

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }

// (hi, lo, delta) -> (hi', lo', 0) with hi' + lo' = hi + lo + delta up to the
// rounding of lo, and hi' the correctly rounded value of the sum.
__device__ __forceinline__ void fold_word(float& hi, float& lo, float& delta)
{
    float s, e;
    two_sum(hi, delta, s, e);
    const float l = __fadd_rn(lo, e);
    const float h = __fadd_rn(s, l);
    lo = __fsub_rn(l, __fsub_rn(h, s));
    hi = h;
    delta = 0.f;
}

// F64 = true: double state; false: float32 compensated state.
// HS (float mode): the hi words of the top level live in shared memory next to
// their lo words, leaving only the per-step delta accumulators in registers;
// this lets one lane own more top words (G = D) within the register file.
template <bool F64, int D, int N, int G, bool HS>
__global__ void __launch_bounds__(kSigWarps * 32, 1)
signature_kernel(const SigArgs a)
{
    using T = typename std::conditional<F64, double, float>::type;
    constexpr int P = N - 2;                 // path levels 1..N-2
    constexpr int SUBS = D / G;              // lanes sharing one level-(N-2) word
    constexpr int64_t W = IPow<D, (P > 0 ? P : 0)>::value * SUBS;  // lanes per stream
    constexpr int TOPW = G * D;              // top words per lane
    static_assert(D % G == 0, "G must divide D");
    // float mode with an even width: top words are updated in f32x2 pairs
    constexpr bool PACK = !F64 && (D % 2 == 0);

    static_assert(!HS || (!F64 && PACK), "hi words in shared memory need the packed float mode");
    // words of top-level state per warp kept in shared memory: lo (float mode),
    // plus hi when HS
    constexpr int TOP_SMEM = F64 ? 0 : (HS ? 2 : 1) * TOPW * 32;

    // dynamic shared memory: [warp][TOP_SMEM] top-level lo (then hi) words,
    // then [warp][kChunk][D] staged increments
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float* lo_top = reinterpret_cast<float*>(smem_raw) + (size_t)warp * TOP_SMEM;
    float2* lo_top2 = reinterpret_cast<float2*>(lo_top);          // packed [TOPW/2][32]
    float2* hi_top2 = reinterpret_cast<float2*>(lo_top + TOPW * 32);  // HS only
    const int nwarps = (int)(blockDim.x >> 5);
    T* xbuf = reinterpret_cast<T*>(smem_raw + (size_t)nwarps * TOP_SMEM * 4) +
              (size_t)warp * kChunk * D;

    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.total_items) break;

        const int64_t slot = item / a.items_per_stream;
        const int64_t blk = item - slot * a.items_per_stream;
        const int64_t s = a.order ? a.order[slot] : slot;
        const int64_t beta_raw = blk * 32 + lane;
        const bool active = beta_raw < W;
        const int64_t beta = active ? beta_raw : (W - 1);
        const int64_t pi = beta / SUBS;
        const int sub = (int)(beta - pi * SUBS);

        int c[P > 0 ? P : 1];
        {
            int64_t t = pi;
#pragma unroll
            for (int i = P - 1; i >= 0; --i) {
                c[i] = (int)(t % D);
                t /= D;
            }
        }

        const int64_t start = a.offsets[s];
        const int64_t len = a.offsets[s + 1] - start;
        const T* __restrict__ xs = static_cast<const T*>(a.inc) + start * D;

        // ---- state
        T ph[P > 0 ? P : 1], mh[G], th[G][D];
        T pd[P > 0 ? P : 1], md[G], td[G][D];   // float mode: delta accumulators
        T pl[P > 0 ? P : 1], ml[G];             // float mode: lo words
#pragma unroll
        for (int i = 0; i < (P > 0 ? P : 1); ++i) ph[i] = pd[i] = pl[i] = T(0);
#pragma unroll
        for (int g = 0; g < G; ++g) {
            mh[g] = md[g] = ml[g] = T(0);
#pragma unroll
            for (int b = 0; b < D; ++b) th[g][b] = td[g][b] = T(0);
        }
        if constexpr (!F64) {
#pragma unroll
            for (int w = 0; w < TOP_SMEM / 32; ++w) lo_top[w * 32 + lane] = 0.f;
        }

        // Increments are staged through shared memory kChunk rows at a time:
        // lane l fetches row t0 + kChunk + l with vector loads while the warp
        // works through rows t0 .. t0 + kChunk - 1, so the global-memory
        // latency is paid once per chunk instead of once per step.
        T nx[D];
        if (lane < len) load_row<T, D>(nx, xs + (int64_t)lane * D);
        int since_fold = 0;
        for (int64_t t0 = 0; t0 < len; t0 += kChunk) {
            __syncwarp();
            if (t0 + lane < len) store_row<T, D>(xbuf + lane * D, nx);
            __syncwarp();
            if (t0 + kChunk + lane < len) load_row<T, D>(nx, xs + (t0 + kChunk + lane) * D);
            const int nsteps = (int)min((int64_t)kChunk, len - t0);
            for (int j = 0; j < nsteps; ++j) {
            const T* row = xbuf + j * D;
            T x[D];
            load_row_smem<T, D>(x, row);
            T xa[G];                               // the lane's letters of level N-1
            load_slice<T, G>(xa, row + sub * G);
            T xc[P > 0 ? P : 1];                   // the lane's path letters
#pragma unroll
            for (int i = 0; i < P; ++i) xc[i] = row[c[i]];

            // pre-step values of the path words (float: hi + delta, hi being
            // kept as the rounded value of hi + lo)
            T vp[P > 0 ? P : 1];
#pragma unroll
            for (int i = 0; i < P; ++i) vp[i] = F64 ? ph[i] : (ph[i] + pd[i]);

            // ---- level N (top): chain through the path, then the mid words
            {
                T acc = T(1);
                if constexpr (P > 0) {
                    acc = vp[0] + xc[0] * (T(1) / T(N));
#pragma unroll
                    for (int i = 2; i <= P; ++i)
                        acc = fma_t(acc, xc[i - 1] * (T(1) / T(N - i + 1)), vp[i - 1]);
                }
                const T accx = acc * (T(1) / T(2));
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    // am = S_{N-1} + acc * x/2; in float mode the delta joins the
                    // product before the (large) hi word
                    const T am = F64 ? fma_t(accx, xa[g], mh[g]) : (mh[g] + fma_t(accx, xa[g], md[g]));
                    if constexpr (PACK) {
                        // packed f32x2 FMAs: two top words per instruction
                        const float2 am2 = make_float2(am, am);
#pragma unroll
                        for (int h = 0; h < D / 2; ++h) {
                            const float2 r = __ffma2_rn(am2, make_float2(x[2 * h], x[2 * h + 1]),
                                                        make_float2(td[g][2 * h], td[g][2 * h + 1]));
                            td[g][2 * h] = r.x;
                            td[g][2 * h + 1] = r.y;
                        }
                    } else {
#pragma unroll
                        for (int b = 0; b < D; ++b) {
                            if constexpr (F64) th[g][b] = fma_t(am, x[b], th[g][b]);
                            else td[g][b] = fma_t(am, x[b], td[g][b]);
                        }
                    }
                }
            }
            // ---- level N-1 (mid words)
            {
                T acc = T(1);
                if constexpr (P > 0) {
                    acc = vp[0] + xc[0] * (T(1) / T(N - 1));
#pragma unroll
                    for (int i = 2; i <= P; ++i)
                        acc = fma_t(acc, xc[i - 1] * (T(1) / T(N - i)), vp[i - 1]);
                }
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    if constexpr (F64) mh[g] = fma_t(acc, xa[g], mh[g]);
                    else md[g] = fma_t(acc, xa[g], md[g]);
                }
            }
            // ---- path levels k = P .. 1
#pragma unroll
            for (int k = P; k >= 1; --k) {
                T upd;
                if (k == 1) {
                    upd = xc[0];
                } else {
                    T acc = vp[0] + xc[0] * (T(1) / T(k));
#pragma unroll
                    for (int i = 2; i <= k - 1; ++i)
                        acc = fma_t(acc, xc[i - 1] * (T(1) / T(k - i + 1)), vp[i - 1]);
                    upd = acc * xc[k - 1];
                }
                if constexpr (F64) ph[k - 1] += upd;
                else pd[k - 1] += upd;
            }

            if constexpr (!F64) {
                if (++since_fold >= a.fold) {
                    since_fold = 0;
                    // Fold the deltas into (hi, lo) with an exact two-sum, then
                    // renormalise (hi, lo) so that hi is the rounded value: the
                    // chains read hi + delta.
#pragma unroll
                    for (int i = 0; i < P; ++i) fold_word(ph[i], pl[i], pd[i]);
#pragma unroll
                    for (int g = 0; g < G; ++g) {
                        fold_word(mh[g], ml[g], md[g]);
                        if constexpr (PACK) {
                            // packed fast two-sum (|hi| >= |delta| except while a word is
                            // still near zero, where the lost error is second order)
#pragma unroll
                            for (int h = 0; h < D / 2; ++h) {
                                float2* hp = hi_top2 + (g * (D / 2) + h) * 32 + lane;
                                const float2 hi = HS ? *hp : make_float2(th[g][2 * h], th[g][2 * h + 1]);
                                const float2 dl = make_float2(td[g][2 * h], td[g][2 * h + 1]);
                                const float2 sm = __fadd2_rn(hi, dl);
                                const float2 z = __ffma2_rn(hi, make_float2(-1.f, -1.f), sm);
                                const float2 er = __ffma2_rn(z, make_float2(-1.f, -1.f), dl);
                                float2* lp = lo_top2 + (g * (D / 2) + h) * 32 + lane;
                                *lp = __fadd2_rn(*lp, er);
                                if constexpr (HS) {
                                    *hp = sm;
                                } else {
                                    th[g][2 * h] = sm.x;
                                    th[g][2 * h + 1] = sm.y;
                                }
                                td[g][2 * h] = 0.f;
                                td[g][2 * h + 1] = 0.f;
                            }
                        } else {
#pragma unroll
                            for (int b = 0; b < D; ++b) {
                                float sh, e;
                                two_sum(th[g][b], td[g][b], sh, e);
                                th[g][b] = sh;
                                float* lp = lo_top + (g * D + b) * 32 + lane;
                                *lp = __fadd_rn(*lp, e);
                                td[g][b] = 0.f;
                            }
                        }
                    }
                }
            }
            }
        }

        // ---- write the stream's words owned by this lane
        if (active) {
            T* __restrict__ o = output_row<T>(a, s);
            if (beta == 0) o[0] = T(1);
            // path words: owned by the lane whose remaining digits are zero
            {
                bool zero_below = (sub == 0);
                int64_t prefix = pi;
#pragma unroll
                for (int k = P; k >= 1; --k) {
                    if (zero_below) {
                        T v;
                        if constexpr (F64) v = ph[k - 1];
                        else v = (ph[k - 1] + (pl[k - 1] + pd[k - 1]));
                        o[a.db[k] + prefix] = v;
                    }
                    zero_below = zero_below && (c[k - 1] == 0);
                    prefix /= D;
                }
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int64_t mw = pi * D + sub * G + g;
                T v;
                if constexpr (F64) v = mh[g];
                else v = mh[g] + (ml[g] + md[g]);
                o[a.db[N - 1] + mw] = v;
#pragma unroll
                for (int b = 0; b < D; ++b) {
                    T tv;
                    if constexpr (F64) tv = th[g][b];
                    else if constexpr (PACK) {
                        const float2 l2 = lo_top2[(g * (D / 2) + b / 2) * 32 + lane];
                        float hv = th[g][b];
                        if constexpr (HS) {
                            const float2 h2 = hi_top2[(g * (D / 2) + b / 2) * 32 + lane];
                            hv = (b & 1) ? h2.y : h2.x;
                        }
                        tv = hv + (((b & 1) ? l2.y : l2.x) + td[g][b]);
                    } else tv = th[g][b] + (lo_top[(g * D + b) * 32 + lane] + td[g][b]);
                    o[a.db[N] + mw * D + b] = tv;
                }
            }
        }
    }
}

// ------------------------------------------------------------------------
// Tensor memory (TMEM) as per-warp storage.  Each SM has 128 lanes x 512
// columns of 32-bit TMEM next to its tensor cores; warp w of a block reads
// and writes lanes 32 (w % 4) .. 32 (w % 4) + 31 with tcgen05.ld / st, one
// lane per thread.  The split kernel below keeps its float64 top-level
// values there instead of in shared memory when `TM` is set (no MMA is
// issued; TMEM only holds state).
__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
}
__device__ __forceinline__ void tmem_st16(uint32_t addr, const uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
        :
        : "r"(addr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]),
          "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]),
          "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM columns a block of nwarps warps takes: 128 per warp in each lane
// quarter (64 float64 values per thread), a power of two
__host__ __device__ constexpr int tmem_cols_for(int nwarps) { return nwarps <= 4 ? 128 : 256; }

// ------------------------------------------------------------------------
// float32 mode on both arithmetic pipes ("split" kernel).
//
// The classic float32 kernel above spends a third of its FP32 pipe on work
// that is not a top-level product: the Horner chains through the path words,
// the path updates, the `hi + delta` reads and the folds.  B200 issues FP64
// instructions to a pipe of their own, so this kernel moves all of that to
// float64 and leaves the FP32 pipe only the products that carry the bulk of
// the work:
//   * path words (levels 1..N-2) are float64 registers updated with DFMAs,
//     and both Horner chains run in float64 from float64 copies of the staged
//     increments; each chain ends in one conversion to float32;
//   * the G mid words (level N-1) keep a float32 delta `md` for the current
//     chunk of kChunk steps and a float64 value in shared memory;
//   * the G*D top words keep a float32 delta `td` per chunk and a float64
//     value in shared memory.
// Within a chunk the top word (w, b) grows by sum_t am_t[w] x_t[b] with
// am_t = S_{N-1}[w] + chain_t * x_t[w]/2, and S_{N-1}[w] = m64 + md_t where
// m64 is the mid word's float64 value at the start of the chunk.  So
//   sum_t am_t x_t[b] = m64 * X[b] + sum_t (md_t + chain_t x_t[w]/2) x_t[b],
// X being the chunk's increment sum: the per-step float32 work is the small
// residual r_t = fma(chain_t/2, x_t[w], md_t) and the products r_t x_t[b]
// (FFMA2), while m64 * X[b] is added in float64 when the chunk's deltas are
// folded (one DFMA per word per chunk).  Per step and lane the FP32 pipe sees
// G*D + 2G FMAs, every one of them a useful Horner FMA.
template <int D, int N, int G, bool TM>
__global__ void __maxnreg__(TM ? RPYB_SIG_TMEM_MAXREG : RPYB_SIG_SPLIT_MAXREG)
signature_kernel_split(const SigArgs a)
{
    constexpr int P = N - 2;                 // path levels 1..N-2
    constexpr int PP = P > 0 ? P : 1;
    constexpr int SUBS = D / G;              // lanes sharing one level-(N-2) word
    constexpr int64_t W = IPow<D, (P > 0 ? P : 0)>::value * SUBS;  // lanes per stream
    constexpr int TOPW = G * D;              // top words per lane
    static_assert(D % G == 0, "G must divide D");
    constexpr bool PACK_T = (D % 2 == 0);    // top words in f32x2 pairs
    constexpr bool PACK_M = (G % 2 == 0);    // mid words in f32x2 pairs

    // dynamic shared memory per warp: top values [TOPW][32] f64 (unless they
    // live in TMEM), mid values [G][32] f64, chunk sums [D] f64 (16-byte
    // padded), staged rows [kChunk][D] f64 then [kChunk][D] f32
    static_assert(!TM || TOPW == 64, "TMEM top level: 64 words per lane (width 8, G = 8)");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    constexpr int TOPS = TM ? 0 : TOPW;     // top words kept in shared memory
    constexpr size_t kXsumBytes = ((size_t)D * 8 + 15) / 16 * 16;
    constexpr size_t kWarpBytes = (size_t)(TOPS + G) * 32 * 8 + kXsumBytes +
                                  (size_t)kChunk * D * 12;
    unsigned char* wbase = smem_raw + (size_t)warp * kWarpBytes;
    double* top64 = reinterpret_cast<double*>(wbase);
    double* mid64 = top64 + TOPS * 32;
    double* xsum = mid64 + G * 32;
    double* x64 = reinterpret_cast<double*>(wbase + (size_t)(TOPS + G) * 32 * 8 + kXsumBytes);
    float* x32 = reinterpret_cast<float*>(x64 + kChunk * D);

    // TMEM for the top level: allocated by warp 0 for the whole block, freed
    // by it after every warp has left the work loop
    __shared__ uint32_t s_tmem_base;
    uint32_t ttop = 0;   // this warp's TMEM address (lane quarter, first column)
    const int nwarps_blk = (int)(blockDim.x >> 5);
    if constexpr (TM) {
        if (warp == 0) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                         :: "r"(smem_u32(&s_tmem_base)), "r"(tmem_cols_for(nwarps_blk)));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        tmem_fence_before();
        __syncthreads();
        tmem_fence_after();
        ttop = s_tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 * (warp >> 2));
    }

    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.total_items) break;

        const int64_t slot = item / a.items_per_stream;
        const int64_t blk = item - slot * a.items_per_stream;
        const int64_t s = a.order ? a.order[slot] : slot;
        const int64_t beta_raw = blk * 32 + lane;
        const bool active = beta_raw < W;
        const int64_t beta = active ? beta_raw : (W - 1);
        const int64_t pi = beta / SUBS;
        const int sub = (int)(beta - pi * SUBS);

        int c[PP];
        {
            int64_t t = pi;
#pragma unroll
            for (int i = P - 1; i >= 0; --i) {
                c[i] = (int)(t % D);
                t /= D;
            }
        }

        const int64_t start = a.offsets[s];
        const int64_t len = a.offsets[s + 1] - start;
        const float* __restrict__ xs = static_cast<const float*>(a.inc) + start * D;

        double ph[PP];
        float md[G], td[G][D];
#pragma unroll
        for (int i = 0; i < PP; ++i) ph[i] = 0.0;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            md[g] = 0.f;
#pragma unroll
            for (int b = 0; b < D; ++b) td[g][b] = 0.f;
        }
#pragma unroll 4
        for (int w = 0; w < TOPS + G; ++w) top64[w * 32 + lane] = 0.0;
        if (lane < D) xsum[lane] = 0.0;
        int chunks_since_fold = 0;
        if constexpr (TM) {
            uint32_t z[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) z[i] = 0u;
#pragma unroll
            for (int q = 0; q < 8; ++q) tmem_st16(ttop + 16 * q, z);
            tmem_wait_st();
        }

        float nx[D];
        if (lane < len) load_row<float, D>(nx, xs + (int64_t)lane * D);
        for (int64_t t0 = 0; t0 < len; t0 += kChunk) {
            const int nsteps = (int)min((int64_t)kChunk, len - t0);
            __syncwarp();
            // stage row t0 + lane in both precisions
            if (lane < nsteps) {
                store_row<float, D>(x32 + lane * D, nx);
                double xd[D];
#pragma unroll
                for (int i = 0; i < D; ++i) xd[i] = (double)nx[i];
                store_row<double, D>(x64 + lane * D, xd);
            }
            __syncwarp();
            if (t0 + kChunk + lane < len) load_row<float, D>(nx, xs + (t0 + kChunk + lane) * D);

            // Software pipeline: the float64 part of step j+1 (its two Horner
            // chains and the path update, which need only the path words after
            // step j) is issued before the float32 products of step j, so the
            // latency of the float64 chain and its conversion hides behind the
            // FFMA2s instead of stalling the warp every step.
            float x[D], accx, accm;
            // chains and path update of step jj: reads the path words before
            // the step, leaves them after it
            auto chains = [&](int jj, float& ax, float& am) {
                const double* row64 = x64 + jj * D;
                double xc[PP];
#pragma unroll
                for (int i = 0; i < P; ++i) xc[i] = row64[c[i]];
                ax = 0.5f;
                am = 1.f;
                if constexpr (P > 0) {
                    double acc = fma(xc[0], 1.0 / N, ph[0]);
#pragma unroll
                    for (int i = 2; i <= P; ++i) acc = fma(acc, xc[i - 1] * (1.0 / (N - i + 1)), ph[i - 1]);
                    ax = (float)(acc * 0.5);
                    double accm64 = fma(xc[0], 1.0 / (N - 1), ph[0]);
#pragma unroll
                    for (int i = 2; i <= P; ++i)
                        accm64 = fma(accm64, xc[i - 1] * (1.0 / (N - i)), ph[i - 1]);
                    am = (float)accm64;
                }
                // path levels k = P .. 1 (top-down: each reads pre-step words)
#pragma unroll
                for (int k = P; k >= 1; --k) {
                    if (k == 1) {
                        ph[0] += xc[0];
                    } else {
                        double acc = fma(xc[0], 1.0 / k, ph[0]);
#pragma unroll
                        for (int i = 2; i <= k - 1; ++i) acc = fma(acc, xc[i - 1] * (1.0 / (k - i + 1)), ph[i - 1]);
                        ph[k - 1] = fma(acc, xc[k - 1], ph[k - 1]);
                    }
                }
            };
            // float32 products of a step: top words, then the mid deltas
            auto products = [&](const float (&xv)[D], float ax, float am) {
                float xa[G];
                if constexpr (SUBS == 1) {
#pragma unroll
                    for (int g = 0; g < G; ++g) xa[g] = xv[g];
                } else {
                    // the lane's G letters of level N-1 (SUBS > 1: a slice of the
                    // row, chosen by selects so that xv stays in registers)
#pragma unroll
                    for (int g = 0; g < G; ++g) xa[g] = xv[g];
#pragma unroll
                    for (int q = 1; q < SUBS; ++q)
#pragma unroll
                        for (int g = 0; g < G; ++g) xa[g] = (sub == q) ? xv[q * G + g] : xa[g];
                }
                float r[G];
                if constexpr (PACK_M) {
#pragma unroll
                    for (int g = 0; g < G; g += 2) {
                        const float2 q = __ffma2_rn(make_float2(ax, ax), make_float2(xa[g], xa[g + 1]),
                                                    make_float2(md[g], md[g + 1]));
                        r[g] = q.x;
                        r[g + 1] = q.y;
                    }
                } else {
#pragma unroll
                    for (int g = 0; g < G; ++g) r[g] = fmaf(ax, xa[g], md[g]);
                }
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    if constexpr (PACK_T) {
                        const float2 r2 = make_float2(r[g], r[g]);
#pragma unroll
                        for (int h = 0; h < D / 2; ++h) {
                            const float2 q = __ffma2_rn(r2, make_float2(xv[2 * h], xv[2 * h + 1]),
                                                        make_float2(td[g][2 * h], td[g][2 * h + 1]));
                            td[g][2 * h] = q.x;
                            td[g][2 * h + 1] = q.y;
                        }
                    } else {
#pragma unroll
                        for (int b = 0; b < D; ++b) td[g][b] = fmaf(r[g], xv[b], td[g][b]);
                    }
                }
                if constexpr (PACK_M) {
#pragma unroll
                    for (int g = 0; g < G; g += 2) {
                        const float2 q = __ffma2_rn(make_float2(am, am), make_float2(xa[g], xa[g + 1]),
                                                    make_float2(md[g], md[g + 1]));
                        md[g] = q.x;
                        md[g + 1] = q.y;
                    }
                } else {
#pragma unroll
                    for (int g = 0; g < G; ++g) md[g] = fmaf(am, xa[g], md[g]);
                }
            };
            // two steps per iteration with alternating register sets, so
            // that the pipeline needs no register copies
            float x1[D], ax1, am1;
            load_row_smem<float, D>(x, x32);
            chains(0, accx, accm);
            int j = 0;
#pragma unroll 1
            for (; j + 2 < nsteps; j += 2) {
                load_row_smem<float, D>(x1, x32 + (j + 1) * D);
                chains(j + 1, ax1, am1);
                products(x, accx, accm);
                load_row_smem<float, D>(x, x32 + (j + 2) * D);
                chains(j + 2, accx, accm);
                products(x1, ax1, am1);
            }
            if (j + 1 < nsteps) {
                load_row_smem<float, D>(x1, x32 + (j + 1) * D);
                chains(j + 1, ax1, am1);
                products(x, accx, accm);
                products(x1, ax1, am1);
            } else {
                products(x, accx, accm);
            }

            // the chunk's increment sum joins the fold period's sum X: with
            // D <= 8 each letter is summed by 32 / 8 = 4 lanes over a quarter
            // of the steps, then the quarters are added by shuffles
            if constexpr (D <= 8) {
                const int letter = lane & 7, quarter = lane >> 3;
                double part = 0.0;
                if (letter < D) {
                    const int j0 = quarter * (kChunk / 4);
#pragma unroll
                    for (int jj = j0; jj < j0 + kChunk / 4; ++jj)
                        if (jj < nsteps) part += x64[jj * D + letter];
                }
                part += __shfl_xor_sync(0xffffffffu, part, 8);
                part += __shfl_xor_sync(0xffffffffu, part, 16);
                if (lane < D) xsum[lane] += part;
            } else if (lane < D) {
                double sum = xsum[lane];
                for (int jj = 0; jj < nsteps; ++jj) sum += x64[jj * D + lane];
                xsum[lane] = sum;
            }
            // ---- fold every fold_chunks chunks and at the stream's end:
            // top += m64 * X + td, mid += md (float64)
            if (++chunks_since_fold < a.fold_chunks && t0 + kChunk < len) continue;
            chunks_since_fold = 0;
            __syncwarp();
            double X[D];
            load_row_smem<double, D>(X, xsum);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                double* mp = mid64 + g * 32 + lane;
                const double m = *mp;
                if constexpr (TM) {
                    // the 8 top words of mid word g: 16 TMEM columns (lo, hi)
                    uint32_t r[16];
                    tmem_ld16(ttop + 16 * g, r);
                    tmem_wait_ld();
#pragma unroll
                    for (int b = 0; b < D; ++b) {
                        double t = __hiloint2double((int)r[2 * b + 1], (int)r[2 * b]);
                        t = fma(m, X[b], t + (double)td[g][b]);
                        r[2 * b] = (uint32_t)__double2loint(t);
                        r[2 * b + 1] = (uint32_t)__double2hiint(t);
                        td[g][b] = 0.f;
                    }
                    tmem_st16(ttop + 16 * g, r);
                } else {
#pragma unroll
                    for (int b = 0; b < D; ++b) {
                        double* tp = top64 + (g * D + b) * 32 + lane;
                        *tp = fma(m, X[b], *tp + (double)td[g][b]);
                        td[g][b] = 0.f;
                    }
                }
                *mp = m + (double)md[g];
                md[g] = 0.f;
            }
            if constexpr (TM) tmem_wait_st();
            __syncwarp();
            if (lane < D) xsum[lane] = 0.0;
        }

        // ---- write the stream's words owned by this lane
        float ttv[TM ? TOPW : 1];
        if constexpr (TM) {
            // warp-wide TMEM reads (every lane takes part, active or not)
#pragma unroll
            for (int g = 0; g < G; ++g) {
                uint32_t r[16];
                tmem_ld16(ttop + 16 * g, r);
                tmem_wait_ld();
#pragma unroll
                for (int b = 0; b < D; ++b)
                    ttv[g * D + b] = (float)__hiloint2double((int)r[2 * b + 1], (int)r[2 * b]);
            }
        }
        if (active) {
            float* __restrict__ o = output_row<float>(a, s);
            if (beta == 0) o[0] = 1.f;
            {
                bool zero_below = (sub == 0);
                int64_t prefix = pi;
#pragma unroll
                for (int k = P; k >= 1; --k) {
                    if (zero_below) o[a.db[k] + prefix] = (float)ph[k - 1];
                    zero_below = zero_below && (c[k - 1] == 0);
                    prefix /= D;
                }
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int64_t mw = pi * D + sub * G + g;
                o[a.db[N - 1] + mw] = (float)mid64[g * 32 + lane];
                float tv[D];
#pragma unroll
                for (int b = 0; b < D; ++b) {
                    if constexpr (TM) tv[b] = ttv[g * D + b];
                    else tv[b] = (float)top64[(g * D + b) * 32 + lane];
                }
                if constexpr (D % 4 == 0) {
                    // a lane's D top words below one mid word are contiguous
                    float* dst = o + a.db[N] + mw * D;
                    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                        store_row<float, D>(dst, tv);
                        continue;
                    }
                }
#pragma unroll
                for (int b = 0; b < D; ++b) o[a.db[N] + mw * D + b] = tv[b];
            }
        }
    }
    if constexpr (TM) {
        tmem_fence_before();
        __syncthreads();
        tmem_fence_after();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                         :: "r"(s_tmem_base), "r"(tmem_cols_for(nwarps_blk)));
    }
}

// ------------------------------------------------------------------------
// Generic fallback for shapes without a specialised instantiation: one warp
// per stream, state as a float64 row in the workspace, levels updated from
// the top down with a warp barrier between levels.
struct GenericTables {
    int64_t db[kMaxDepth + 2];
    int64_t pw[kMaxDepth + 1];
};

__global__ void signature_generic_kernel(int mode, int d, int n, const int64_t* offsets,
                                         const void* inc, void* out, int64_t ld_out,
                                         int64_t n_streams, double* state, int64_t T,
                                         const GenericTables tab)
{
    const int64_t* db = tab.db;
    const int64_t* pw = tab.pw;
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = wid; s < n_streams; s += nw) {
        double* S = state + s * T;
        for (int64_t i = lane; i < T; i += 32) S[i] = (i == 0) ? 1.0 : 0.0;
        __syncwarp();
        const int64_t start = offsets[s], len = offsets[s + 1] - start;
        for (int64_t t = 0; t < len; ++t) {
            const int64_t rowoff = (start + t) * d;
            for (int k = n; k >= 1; --k) {
                for (int64_t w = lane; w < pw[k]; w += 32) {
                    // Horner over the prefixes of w: acc_i = S_i[w_1..w_i] + acc_{i-1} x[w_i]/(k-i+1)
                    double acc = 1.0;
                    for (int i = 1; i <= k; ++i) {
                        const int64_t pref = w / pw[k - i];
                        const int letter = (int)(pref % d);
                        const double xv = (mode == RPYB_F64)
                                              ? static_cast<const double*>(inc)[rowoff + letter]
                                              : (double)static_cast<const float*>(inc)[rowoff + letter];
                        const double scaled = acc * xv / (double)(k - i + 1);
                        if (i < k) acc = S[db[i] + pref] + scaled;
                        else acc = scaled;
                    }
                    S[db[k] + w] += acc;
                }
                __syncwarp();
            }
        }
        for (int64_t i = lane; i < T; i += 32) {
            if (mode == RPYB_F64) static_cast<double*>(out)[s * ld_out + i] = S[i];
            else static_cast<float*>(out)[s * ld_out + i] = (float)S[i];
        }
        __syncwarp();
    }
}

using SigKernel = void (*)(SigArgs);

struct SigVariant {
    SigKernel fn;
    int g;
    int64_t lanes;          // W: lanes per stream
    size_t smem_warp;       // dynamic shared memory per warp (bytes)
    bool tmem = false;      // top level in TMEM: blocks of at most 4 warps, 4 blocks per SM
};

template <bool F64, int D, int N, int G, bool HS>
SigVariant make_variant()
{
    constexpr int64_t W = IPow<D, N - 2>::value * (D / G);
    constexpr size_t top = F64 ? 0 : (size_t)(HS ? 2 : 1) * G * D * 32 * 4;
    constexpr size_t stage = (size_t)kChunk * D * (F64 ? 8 : 4);
    return SigVariant{&signature_kernel<F64, D, N, G, HS>, G, W, top + stage};
}

template <int D, int N, int G, bool TM = false>
SigVariant make_split_variant()
{
    constexpr int64_t W = IPow<D, N - 2>::value * (D / G);
    constexpr size_t xsum = ((size_t)D * 8 + 15) / 16 * 16;
    constexpr size_t bytes = (size_t)((TM ? 0 : G * D) + G) * 32 * 8 + xsum + (size_t)kChunk * D * 12;
    return SigVariant{&signature_kernel_split<D, N, G, TM>, G, W, bytes, TM};
}

// The split kernel's top level in TMEM at width 8 (RPYB_SIG_TMEM=1).  Off by
// default: measured on B200 at 12 resident warps it was within 2 % of the
// shared-memory layout at 8, because the kernel is bound by its arithmetic
// pipes rather than by occupancy.
bool split_tmem_enabled()
{
    static const bool on = [] {
        const char* e = getenv("RPYB_SIG_TMEM");
        return e && e[0] == '1';
    }();
    return on;
}

template <bool F64, int D, int G, bool HS>
bool pick_depth(int n, SigVariant& v)
{
    switch (n) {
        case 2: v = make_variant<F64, D, 2, G, HS>(); return true;
        case 3: v = make_variant<F64, D, 3, G, HS>(); return true;
        case 4: v = make_variant<F64, D, 4, G, HS>(); return true;
        case 5: v = make_variant<F64, D, 5, G, HS>(); return true;
        case 6: v = make_variant<F64, D, 6, G, HS>(); return true;
        case 7:
            if constexpr (D <= 4) { v = make_variant<F64, D, 7, G, HS>(); return true; }
            return false;
        case 8:
            if constexpr (D <= 3) { v = make_variant<F64, D, 8, G, HS>(); return true; }
            return false;
        default: return false;
    }
}

template <int D, int G>
bool pick_split_depth(int n, SigVariant& v)
{
    if constexpr (D == 8 && G == 8) {
        if (split_tmem_enabled()) {
            switch (n) {
                case 2: v = make_split_variant<D, 2, G, true>(); return true;
                case 3: v = make_split_variant<D, 3, G, true>(); return true;
                case 4: v = make_split_variant<D, 4, G, true>(); return true;
                case 5: v = make_split_variant<D, 5, G, true>(); return true;
                case 6: v = make_split_variant<D, 6, G, true>(); return true;
                default: return false;
            }
        }
    }
    switch (n) {
        case 2: v = make_split_variant<D, 2, G>(); return true;
        case 3: v = make_split_variant<D, 3, G>(); return true;
        case 4: v = make_split_variant<D, 4, G>(); return true;
        case 5: v = make_split_variant<D, 5, G>(); return true;
        case 6: v = make_split_variant<D, 6, G>(); return true;
        case 7:
            if constexpr (D <= 4) { v = make_split_variant<D, 7, G>(); return true; }
            return false;
        case 8:
            if constexpr (D <= 3) { v = make_split_variant<D, 8, G>(); return true; }
            return false;
        default: return false;
    }
}

// Kernel families of the specialised path.
enum SigFamily { kFamilyClassic = 0, kFamilySplit = 1 };

// Lane shapes: G level-(N-1) words (and G*D top words) per lane.  The first
// entry of each list is the default; the others are the autotuner's
// alternatives.  G only decides how a stream's words are dealt to lanes:
// every word sees the same arithmetic whatever G is, so the alternatives
// give bitwise identical results.
//  - float64: G words of double state per lane;
//  - classic float32: at width 8 the top-level hi words live in shared
//    memory so that one lane can own all 64 top words below its word;
//  - split float32: G*D float32 deltas per lane.
bool lane_shapes(int mode, int family, int d, int* gs, int* count)
{
    *count = 0;
    auto put = [&](std::initializer_list<int> l) { for (int g : l) gs[(*count)++] = g; };
    if (mode == RPYB_F64) {
        switch (d) {
            case 2: put({2}); break;
            case 3: put({3}); break;
            case 4: put({4, 2}); break;
            case 5: put({5}); break;
            case 6: put({3, 6}); break;
            case 7: put({7}); break;
            case 8: put({RPYB_SIG_F64_G8, RPYB_SIG_F64_G8 == 8 ? 4 : 8}); break;
            default: return false;
        }
    } else if (family == kFamilyClassic) {
        switch (d) {
            case 2: put({2}); break;
            case 3: put({3}); break;
            case 4: put({4}); break;
            case 5: put({5}); break;
            case 6: put({3}); break;
            case 7: put({7}); break;
            case 8: put({8}); break;
            default: return false;
        }
    } else {
        switch (d) {
            case 2: put({2}); break;
            case 3: put({3}); break;
            case 4: put({4, 2}); break;
            case 5: put({5}); break;
            case 6: put({6, 3}); break;
            case 7: put({7}); break;
            case 8: put({8, 4}); break;
            default: return false;
        }
    }
    return true;
}

bool pick_f64(int d, int n, int g, SigVariant& v)
{
    switch (d * 16 + g) {
        case 2 * 16 + 2: return pick_depth<true, 2, 2, false>(n, v);
        case 3 * 16 + 3: return pick_depth<true, 3, 3, false>(n, v);
        case 4 * 16 + 4: return pick_depth<true, 4, 4, false>(n, v);
        case 4 * 16 + 2: return pick_depth<true, 4, 2, false>(n, v);
        case 5 * 16 + 5: return pick_depth<true, 5, 5, false>(n, v);
        case 6 * 16 + 3: return pick_depth<true, 6, 3, false>(n, v);
        case 6 * 16 + 6: return pick_depth<true, 6, 6, false>(n, v);
        case 7 * 16 + 7: return pick_depth<true, 7, 7, false>(n, v);
        case 8 * 16 + 8: return pick_depth<true, 8, 8, false>(n, v);
        case 8 * 16 + 4: return pick_depth<true, 8, 4, false>(n, v);
        default: return false;
    }
}

bool pick_classic_f32(int d, int n, int g, SigVariant& v)
{
    switch (d * 16 + g) {
        case 2 * 16 + 2: return pick_depth<false, 2, 2, false>(n, v);
        case 3 * 16 + 3: return pick_depth<false, 3, 3, false>(n, v);
        case 4 * 16 + 4: return pick_depth<false, 4, 4, false>(n, v);
        case 5 * 16 + 5: return pick_depth<false, 5, 5, false>(n, v);
        case 6 * 16 + 3: return pick_depth<false, 6, 3, false>(n, v);
        case 7 * 16 + 7: return pick_depth<false, 7, 7, false>(n, v);
        case 8 * 16 + 8: return pick_depth<false, 8, 8, true>(n, v);
        default: return false;
    }
}

bool pick_split(int d, int n, int g, SigVariant& v)
{
    switch (d * 16 + g) {
        case 2 * 16 + 2: return pick_split_depth<2, 2>(n, v);
        case 3 * 16 + 3: return pick_split_depth<3, 3>(n, v);
        case 4 * 16 + 4: return pick_split_depth<4, 4>(n, v);
        case 4 * 16 + 2: return pick_split_depth<4, 2>(n, v);
        case 5 * 16 + 5: return pick_split_depth<5, 5>(n, v);
        case 6 * 16 + 6: return pick_split_depth<6, 6>(n, v);
        case 6 * 16 + 3: return pick_split_depth<6, 3>(n, v);
        case 7 * 16 + 7: return pick_split_depth<7, 7>(n, v);
        case 8 * 16 + 8: return pick_split_depth<8, 8>(n, v);
        case 8 * 16 + 4: return pick_split_depth<8, 4>(n, v);
        default: return false;
    }
}

// Default float32 family: RPYB_SIG_F32_KERNEL=classic selects the
// single-pipe compensated kernel, anything else the split kernel.
int default_f32_family()
{
    static int fam = [] {
        const char* e = getenv("RPYB_SIG_F32_KERNEL");
        return (e && std::string(e) == "classic") ? kFamilyClassic : kFamilySplit;
    }();
    return fam;
}

// The specialised kernel for (mode, family, width, depth, G); g == 0 takes
// the default lane shape.  Returns false for shapes served by the generic
// kernel.
bool pick_signature_variant(int mode, int family, int d, int n, int g, SigVariant& v)
{
    if (n < 2) return false;
    int gs[4], count = 0;
    if (!lane_shapes(mode, family, d, gs, &count)) return false;
    if (g == 0) g = gs[0];
    if (mode == RPYB_F64) return pick_f64(d, n, g, v);
    if (family == kFamilyClassic) return pick_classic_f32(d, n, g, v);
    return pick_split(d, n, g, v);
}

bool pick_signature_variant(int mode, int d, int n, SigVariant& v)
{
    return pick_signature_variant(mode, mode == RPYB_F64 ? kFamilyClassic : default_f32_family(),
                                  d, n, 0, v);
}

// Widens float32 increment rows to float64 (the reference run of the
// error report computes from the same float32 inputs).
__global__ void widen_rows_kernel(const float* __restrict__ in, double* __restrict__ out, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

// err[s] = max over levels k of ||got_k - ref_k||_inf / ||ref_k||_inf for
// stream s (the absolute difference where the reference level is zero).
// One block per stream, levels reduced in shared memory.
__global__ void level_error_kernel(const float* __restrict__ got, int64_t ld_got,
                                   const double* __restrict__ ref, int64_t ld_ref, int depth,
                                   const GenericTables tab, double* __restrict__ err, int64_t n)
{
    __shared__ double s_num[32], s_den[32];
    for (int64_t s = blockIdx.x; s < n; s += gridDim.x) {
        const float* g = got + s * ld_got;
        const double* r = ref + s * ld_ref;
        double worst = 0.0;
        for (int k = 0; k <= depth; ++k) {
            double num = 0.0, den = 0.0;
            for (int64_t i = tab.db[k] + threadIdx.x; i < tab.db[k + 1]; i += blockDim.x) {
                const double rv = r[i];
                num = fmax(num, fabs((double)g[i] - rv));
                den = fmax(den, fabs(rv));
            }
            for (int o = 16; o > 0; o >>= 1) {
                num = fmax(num, __shfl_xor_sync(0xffffffffu, num, o));
                den = fmax(den, __shfl_xor_sync(0xffffffffu, den, o));
            }
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            __syncthreads();
            if (lane == 0) {
                s_num[warp] = num;
                s_den[warp] = den;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
                    num = fmax(num, s_num[w]);
                    den = fmax(den, s_den[w]);
                }
                worst = fmax(worst, den > 0.0 ? num / den : num);
            }
        }
        if (threadIdx.x == 0) err[s] = worst;
        __syncthreads();
    }
}

int device_sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 148;
    return sms;
}

}  // namespace

int signature_warps_per_block()
{
    static int wpb = [] {
        // 0 = choose by occupancy; RPYB_SIG_WPB forces a block size
        const char* e = getenv("RPYB_SIG_WPB");
        int w = e ? atoi(e) : 0;
        return (w >= 1 && w <= kSigWarps) ? w : 0;
    }();
    return wpb;
}

int signature_fold_interval()
{
    static int fold = [] {
        const char* e = getenv("RPYB_SIG_FOLD");
        int f = e ? atoi(e) : 24;
        return f > 0 ? f : 24;
    }();
    return fold;
}

// Chunks of 32 steps between the split kernel's folds (RPYB_SIG_SPLIT_FOLD).
// Measured on B200 on the 4096-stream width-8 depth-5 workload (time, max
// error against float64): 2 -> 17.45 ms, 7.6e-7; 3 -> 16.86 ms, 7.3e-7;
// 4 -> 16.72 ms, 1.03e-6 (over the 1e-6 bar).
int split_fold_chunks()
{
    static int f = [] {
        const char* e = getenv("RPYB_SIG_SPLIT_FOLD");
        const int v = e ? atoi(e) : 3;
        return (v >= 1 && v <= 64) ? v : 3;
    }();
    return f;
}

namespace {

// One launch of a specialised signature kernel over n_items work streams
// (streams, or the time segments of split streams).  `queue` is a zeroed-on-
// launch device counter of the workspace.  wpb = 0 chooses the block size by
// occupancy (RPYB_SIG_WPB overrides).  The kernel attribute and the block
// size are fixed once per device, kernel, per-warp shared memory and forced
// block size, so repeated launches (and a launch captured into a CUDA graph)
// only reset the queue and launch.
int launch_signature_variant(const SigVariant& v, const Geometry& g, int64_t n_items,
                             const int64_t* offsets, const void* inc, void* out, int64_t ld_out,
                             const int64_t* order, const int64_t* dst_row, void* alt,
                             int64_t ld_alt, int* queue, int wpb_forced, cudaStream_t s)
{
    SigArgs a{};
    a.offsets = offsets;
    a.inc = inc;
    a.out = out;
    a.ld_out = ld_out;
    a.order = order;
    a.n_streams = n_items;
    a.items_per_stream = (v.lanes + 31) / 32;
    a.total_items = a.items_per_stream * n_items;
    if (a.total_items > 0x7fffffff) return fail(RPYB_E_UNSUPPORTED, "too many work items");
    a.queue = queue;
    a.fold = signature_fold_interval();
    a.fold_chunks = split_fold_chunks();
    a.dst_row = dst_row;
    a.alt = alt;
    a.ld_alt = ld_alt;
    for (int k = 0; k <= kMaxDepth + 1; ++k) a.db[k] = g.db[k];
    const size_t smem_warp = v.smem_warp;
    int wpb = signature_warps_per_block();
    if (wpb == 0) wpb = (wpb_forced >= 1 && wpb_forced <= kSigWarps) ? wpb_forced : 0;
    int per_sm = 0;
    {
        static std::mutex mu;
        static std::map<std::tuple<int, const void*, size_t, int>, std::pair<int, int>> chosen;
        int dev = 0;
        RPYB_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(mu);
        const auto key = std::make_tuple(dev, (const void*)v.fn, smem_warp, wpb);
        auto it = chosen.find(key);
        if (it == chosen.end()) {
            RPYB_CUDA(cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(smem_warp * kSigWarps)));
            // the whole unified L1/shared array as shared memory: the kernels
            // stage their state there and read global memory once per chunk
            RPYB_CUDA(cudaFuncSetAttribute(v.fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared));
            int best_wpb = wpb, best_per_sm = 0;
            if (wpb == 0) {
                // warps are independent: the block size only matters for
                // occupancy, so take the one fitting the most warps per SM
                // (TMEM variants: blocks of up to 4 warps, 4 blocks per SM,
                // so that the blocks' TMEM never exceeds the SM's 512 columns)
                int best_warps = -1;
                for (int w = v.tmem ? 4 : kSigWarps; w >= 1; --w) {
                    int bps = 0;
                    RPYB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, v.fn, w * 32,
                                                                            smem_warp * w));
                    if (v.tmem) bps = std::min(bps, 512 / tmem_cols_for(w));
                    if (bps * w > best_warps) {
                        best_warps = bps * w;
                        best_wpb = w;
                        best_per_sm = bps;
                    }
                }
            } else {
                RPYB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&best_per_sm, v.fn,
                                                                        wpb * 32, smem_warp * wpb));
                if (v.tmem) best_per_sm = std::min(best_per_sm, 512 / tmem_cols_for(wpb));
            }
            it = chosen.emplace(key, std::make_pair(best_wpb, best_per_sm)).first;
        }
        wpb = it->second.first;
        per_sm = it->second.second;
    }
    {
        // RPYB_SIG_BLOCKS_PER_SM forces the resident blocks per SM the grid
        // is sized for (the occupancy calculator's figure otherwise)
        static const int forced_bps = [] {
            const char* e = getenv("RPYB_SIG_BLOCKS_PER_SM");
            const int b = e ? atoi(e) : 0;
            return (b >= 1 && b <= 32) ? b : 0;
        }();
        if (forced_bps) per_sm = v.tmem ? std::min(forced_bps, 512 / tmem_cols_for(wpb)) : forced_bps;
    }
    if (per_sm < 1) per_sm = 1;
    const size_t smem = smem_warp * wpb;
    int64_t blocks = (int64_t)per_sm * device_sm_count();
    blocks = std::min<int64_t>(blocks, (a.total_items + wpb - 1) / wpb);
    if (blocks < 1) blocks = 1;
    RPYB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), s));
    v.fn<<<(unsigned)blocks, wpb * 32, smem, s>>>(a);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

}  // namespace

bool signature_lane_shapes(int mode, int width, int depth, int* gs, int* count)
{
    SigVariant v;
    if (!pick_signature_variant(mode, width, depth, v)) return false;
    return lane_shapes(mode, mode == RPYB_F64 ? kFamilyClassic : default_f32_family(), width, gs,
                       count);
}

int64_t signature_lanes_per_stream(int mode, int width, int depth, int g)
{
    SigVariant v;
    const int family = mode == RPYB_F64 ? kFamilyClassic : default_f32_family();
    if (!pick_signature_variant(mode, family, width, depth, g, v)) return -1;
    return v.lanes;
}

int signature_launch(int mode, int width, int depth, int g_lane, int wpb, int64_t n_items,
                     const int64_t* offsets, const void* inc, void* out, int64_t ld_out,
                     const int64_t* order, const int64_t* dst_row, void* alt, int64_t ld_alt,
                     int* queue, cudaStream_t s)
{
    int rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    SigVariant v;
    const int family = mode == RPYB_F64 ? kFamilyClassic : default_f32_family();
    if (!pick_signature_variant(mode, family, width, depth, g_lane, v))
        return fail(RPYB_E_UNSUPPORTED, "no specialised signature kernel for this shape");
    if (n_items == 0) return RPYB_OK;
    const bool vec = (mode == RPYB_F32) ? (width % 4 == 0) : (width % 2 == 0);
    if (vec && (reinterpret_cast<uintptr_t>(inc) & 15) != 0)
        return fail(RPYB_E_INVALID, "increments must be 16-byte aligned");
    return launch_signature_variant(v, g, n_items, offsets, inc, out, ld_out, order, dst_row, alt,
                                    ld_alt, queue, wpb, s);
}

int signature_error_report(int width, int depth, int64_t n_streams, const int64_t* offsets,
                           const void* inc32, int64_t total_rows, const void* out32,
                           int64_t ld_out, const int64_t* order, double* err_out, void* ws,
                           size_t ws_bytes, cudaStream_t s)
{
    int rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    auto up = [](int64_t b) { return (b + 255) / 256 * 256; };
    const int64_t T = g.size();
    const int64_t base = up(rpyb_signature_workspace_size(RPYB_F32, width, depth, n_streams));
    const int64_t refws = up(rpyb_signature_workspace_size(RPYB_F64, width, depth, n_streams));
    const int64_t refout = up(n_streams * T * 8);
    const int64_t need = base + refws + refout + up(total_rows * width * 8);
    if ((int64_t)ws_bytes < need) return fail(RPYB_E_NOMEM, "error-report workspace too small");
    char* w0 = static_cast<char*>(ws);
    double* ref = reinterpret_cast<double*>(w0 + base + refws);
    double* inc64 = reinterpret_cast<double*>(w0 + base + refws + refout);
    const int64_t nval = total_rows * width;
    if (nval > 0) {
        const int64_t blocks = std::min<int64_t>((nval + 255) / 256, 4096);
        widen_rows_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<const float*>(inc32),
                                                           inc64, nval);
        RPYB_CUDA(cudaGetLastError());
    }
    if ((rc = rpyb_signature(RPYB_F64, width, depth, n_streams, offsets, inc64, ref, T, order,
                             w0 + base, (size_t)refws, s)))
        return rc;
    GenericTables tab{};
    for (int k = 0; k < kMaxDepth + 2; ++k) tab.db[k] = g.db[k];
    const int64_t blocks = std::min<int64_t>(n_streams, (int64_t)device_sm_count() * 8);
    level_error_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, s>>>(
        static_cast<const float*>(out32), ld_out, ref, T, depth, tab, err_out, n_streams);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_signature_workspace_size(int mode, int32_t width, int32_t depth,
                                               int64_t n_streams)
{
    Geometry g;
    if (make_geometry(width, depth, g)) return -1;
    SigVariant v;
    const bool special = pick_signature_variant(mode, width, depth, v);
    int64_t bytes = 256;  // queue counter
    if (!special) bytes += n_streams * g.size() * 8;
    return bytes;
}

RPYB_API int rpyb_signature(int mode, int32_t width, int32_t depth, int64_t n_streams,
                            const int64_t* offsets, const void* increments, void* out,
                            int64_t ld_out, const int64_t* order, void* workspace,
                            size_t workspace_bytes, void* stream)
{
    int rc;
    if (mode != RPYB_F32 && mode != RPYB_F64)
        return fail(RPYB_E_INVALID, "unsupported signature mode");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n_streams < 0) return fail(RPYB_E_INVALID, "negative number of streams");
    if (n_streams == 0) return RPYB_OK;
    if (!offsets || !out) return fail(RPYB_E_INVALID, "null pointer");
    if (n_streams > 1 && ld_out < g.size()) return fail(RPYB_E_INVALID, "ld_out too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t need = rpyb_signature_workspace_size(mode, width, depth, n_streams);
    Scratch scratch(workspace, workspace_bytes, s);
    void* ws = nullptr;
    if ((rc = scratch.get((size_t)need, &ws))) return rc;

    SigVariant v{};
    const bool special = pick_signature_variant(mode, width, depth, v);
    if (special) {
        if (increments == nullptr) return fail(RPYB_E_INVALID, "null increments");
        const bool vec = (mode == RPYB_F32) ? (width % 4 == 0) : (width % 2 == 0);
        if (vec && (reinterpret_cast<uintptr_t>(increments) & 15) != 0)
            return fail(RPYB_E_INVALID, "increments must be 16-byte aligned");
        return launch_signature_variant(v, g, n_streams, offsets, increments, out, ld_out, order,
                                        nullptr, nullptr, 0, static_cast<int*>(ws), 0, s);
    }
    // generic path
    const int sms = device_sm_count();
    double* state = reinterpret_cast<double*>(static_cast<char*>(ws) + 256);
    GenericTables tab;
    for (int k = 0; k < kMaxDepth + 2; ++k) tab.db[k] = g.db[k];
    for (int k = 0; k <= kMaxDepth; ++k) tab.pw[k] = g.pw[k];
    const int64_t warps = std::min<int64_t>(n_streams, (int64_t)sms * 16);
    const int threads = 128;
    const int64_t blocks = (warps * 32 + threads - 1) / threads;
    signature_generic_kernel<<<(unsigned)blocks, threads, 0, s>>>(
        mode, width, depth, offsets, increments, out, ld_out, n_streams, state, g.size(), tab);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

RPYB_API int64_t rpyb_signature_batched_workspace_size(int mode, int32_t width, int32_t depth,
                                                       int64_t n_streams, int64_t total_rows,
                                                       int with_error)
{
    const int64_t base = rpyb_signature_workspace_size(mode, width, depth, n_streams);
    if (base < 0 || n_streams < 0 || total_rows < 0) return -1;
    if (!with_error || mode != RPYB_F32) return base;
    auto up = [](int64_t b) { return (b + 255) / 256 * 256; };
    const int64_t T = rpyb_tensor_size(width, depth);
    const int64_t ref = rpyb_signature_workspace_size(RPYB_F64, width, depth, n_streams);
    return up(base) + up(ref) + up(n_streams * T * 8) + up(total_rows * width * 8);
}

RPYB_API int rpyb_signature_batched(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                    const int64_t* offsets, const void* increments,
                                    int64_t total_rows, void* out, int64_t ld_out,
                                    const int64_t* order, double* err_out, void* workspace,
                                    size_t workspace_bytes, void* stream)
{
    int rc;
    if (mode != RPYB_F32 && mode != RPYB_F64)
        return fail(RPYB_E_INVALID, "unsupported signature mode");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n_streams < 0 || total_rows < 0) return fail(RPYB_E_INVALID, "negative size");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (err_out == nullptr) {
        return rpyb_signature(mode, width, depth, n_streams, offsets, increments, out, ld_out,
                              order, workspace, workspace_bytes, stream);
    }
    if (n_streams == 0) return RPYB_OK;
    if (mode == RPYB_F64) {
        // the float64 path is its own reference
        if ((rc = rpyb_signature(mode, width, depth, n_streams, offsets, increments, out, ld_out,
                                 order, workspace, workspace_bytes, stream)))
            return rc;
        RPYB_CUDA(cudaMemsetAsync(err_out, 0, (size_t)n_streams * sizeof(double), s));
        return RPYB_OK;
    }
    if (total_rows > 0 && increments == nullptr) return fail(RPYB_E_INVALID, "null increments");
    const int64_t need = rpyb_signature_batched_workspace_size(mode, width, depth, n_streams,
                                                               total_rows, 1);
    Scratch scratch(workspace, workspace_bytes, s);
    void* ws = nullptr;
    if ((rc = scratch.get((size_t)need, &ws))) return rc;
    // with no rows at all the kernels read no increment; any aligned pointer will do
    const void* inc32 = (total_rows > 0) ? increments : static_cast<const void*>(ws);
    const int64_t base = (rpyb_signature_workspace_size(mode, width, depth, n_streams) + 255) /
                         256 * 256;
    if ((rc = rpyb_signature(RPYB_F32, width, depth, n_streams, offsets, inc32, out, ld_out,
                             order, ws, (size_t)base, stream)))
        return rc;
    return signature_error_report(width, depth, n_streams, offsets, inc32, total_rows, out,
                                  ld_out, order, err_out, ws, (size_t)need, s);
}

}  // extern "C"
