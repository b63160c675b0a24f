// Reverse-mode derivative of batched signatures (the signature adjoint).
//
// For S_{t+1} = S_t (x) exp(x_t) and an upstream gradient G_L = dLoss/dS_L
// (e.g. W for Loss = <W, S_L>), the reverse pass walks every stream backwards
// and produces dLoss/dx_t and G_t = dLoss/dS_t from G_{t+1}.  Two facts shape
// the kernels:
//
//   * G_t = exp(D_x) G_{t+1}, where D_x contracts the last letter of a word
//     with x:  (D_x G)[u] = sum_a x_a G[u a].  It only moves adjoint mass
//     from longer words to their prefixes, so the top level of G never
//     changes and every subtree's adjoint evolves on its own.  Writing
//     M_q[u] = sum_{|v|=q} x^v G_{t+1}[u v], level k of G_t is
//     sum_q M_q / q!.
//   * dLoss/dx_a = sum_w sum_q F_q(w) M_q(w a), where
//     F_q(w) = sum_p S_t[w_1..w_{|w|-p}] x^{last p letters of w} / (p+q+1)!
//     is the Horner chain of the forward step with shifted divisors, built
//     from S_t at the prefixes of w (levels <= N-1 only).
//
// Lane kernel (widths 2..8 with width^(depth-2) <= 992): one block per
// stream, one thread ("lane") per level-(N-2) word pi.  A lane keeps S_t on
// its prefix path and on pi's D children (levels <= N-1; the top level of S
// is never needed) and G on pi in float64 registers, and G on pi's children
// in shared memory next to the constant top level of G.  S_t is recovered from
// S_{t+1} by the inverse step S_t = S_{t+1} (x) exp(-x_t) and re-anchored to
// a forward checkpoint every K steps.  The lanes' subtree terms need no
// communication.  Up to four extra "fold" warps per block trail the lanes by
// a step: they fold the adjoints of the shared ancestors (levels 1..N-3)
// level by level and sum the step's gradient (lane partials come pre-reduced
// by a warp reduce-scatter).  Lanes and fold warps hand buffers over through
// named barriers (bar.arrive / bar.sync), so the lanes wait for the folding
// only when they run NB steps ahead.
//
// Block kernel (every other shape): one block per stream walks all words of
// the tensor in global memory:
//   * checkpoint pass: S_t is propagated forwards in float64 and stored every
//     K steps;
//   * per segment (last first): the K states of the segment are recomputed
//     from its checkpoint, then for t = segment end .. segment start the step
//     is differentiated through its Horner chains
//       acc_1 = S_1 + x/k, acc_i = S_i + acc_{i-1} (x) x/(k-i+1),
//       S'_k  = S_k + acc_{k-1} (x) x.
//
// The reference has no reverse-mode derivative (its sig_derivative is
// forward mode, algebra/src/lite_context.h:577-636); results are checked
// against float64 autograd, central finite differences and that forward
// derivative.
//
// Precision: adjoint accumulators and states are float64 in both modes; in
// mode RPYB_F32 the top-level products (the bulk of the work) and the lanes'
// per-step gradient partials are float32.
#include <algorithm>
#include <climits>
#include <string>

#include "common.cuh"

namespace rpyb {
namespace {

constexpr int kBwdThreads = 512;

struct BwdArgs {
    int width, depth;
    int64_t n_streams;
    const int64_t* offsets;
    const void* inc;
    const void* grad_sig;
    int64_t ld_grad;           // 0: one gradient row shared by every stream
    void* grad_inc;
    int K;                     // checkpoint interval
    int64_t max_segments;      // ceil(max len / K)
    int64_t T;
    int64_t db[kMaxDepth + 2];
    int64_t pw[kMaxDepth + 1];
    int* queue;
    char* scratch;
    int64_t slot_bytes;
};

template <typename T>
__device__ __forceinline__ T ld_inc(const void* p, int64_t i)
{
    return static_cast<const T*>(p)[i];
}

// new = S (x) exp(x) for every word (levels 1..N), prefix-chain formula per
// word; S and new are distinct buffers.  x holds the D letters (type U).
template <typename U, int D>
__device__ void step_forward(const BwdArgs& a, const U* __restrict__ S, U* __restrict__ out,
                             const U (&x)[D])
{
    const int N = a.depth;
    for (int64_t e = threadIdx.x; e < a.T; e += blockDim.x) {
        if (e == 0) {
            out[0] = S[0];
            continue;
        }
        int k = 1;
        while (e >= a.db[k + 1]) ++k;
        const int64_t w = e - a.db[k];
        U acc = U(1);
        for (int i = 1; i < k; ++i) {
            const int64_t pref = w / a.pw[k - i];
            const int letter = (int)(pref % D);
            acc = S[a.db[i] + pref] + acc * x[letter] / U(k - i + 1);
        }
        out[e] = S[e] + acc * x[(int)(w % D)];
    }
    (void)N;
}

template <typename T, int D>
__global__ void __launch_bounds__(kBwdThreads)
signature_backward_kernel(const BwdArgs a)
{
    using U = T;                                   // state/chain arithmetic type
    __shared__ int s_item;
    __shared__ double s_red[kBwdThreads / 32][D];

    char* slot = a.scratch + (int64_t)blockIdx.x * a.slot_bytes;
    const int64_t T_ = a.T;
    double* G = reinterpret_cast<double*>(slot);                 // T
    double* abar = G + T_;                                       // T
    double* fwd0 = abar + T_;                                    // T (checkpoint pass)
    double* fwd1 = fwd0 + T_;                                    // T
    U* chain = reinterpret_cast<U*>(fwd1 + T_);                  // T
    U* states = chain + T_;                                      // K * T
    U* ckpt = states + (int64_t)a.K * T_;                        // max_segments * T

    const int N = a.depth;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(a.queue, 1);
        __syncthreads();
        const int64_t s = s_item;
        __syncthreads();
        if (s >= a.n_streams) break;
        const int64_t start = a.offsets[s];
        const int64_t len = a.offsets[s + 1] - start;
        const int64_t nseg = (len + a.K - 1) / a.K;
        if (nseg > a.max_segments) {
            // unreachable: the host rejects batches whose longest stream
            // exceeds max_len before launching; kept as a guard so that a
            // stream without checkpoint scratch never writes past its slot
            for (int64_t e = threadIdx.x; e < len * D; e += blockDim.x)
                static_cast<T*>(a.grad_inc)[start * D + e] = (T)NAN;
            continue;
        }

        // ---- checkpoint pass (float64)
        for (int64_t e = threadIdx.x; e < T_; e += blockDim.x) fwd0[e] = (e == 0) ? 1.0 : 0.0;
        __syncthreads();
        double* cur = fwd0;
        double* nxt = fwd1;
        for (int64_t t = 0; t < len; ++t) {
            if (t % a.K == 0) {
                U* row = ckpt + (t / a.K) * T_;
                for (int64_t e = threadIdx.x; e < T_; e += blockDim.x) row[e] = (U)cur[e];
            }
            double x[D];
#pragma unroll
            for (int c = 0; c < D; ++c) x[c] = (double)ld_inc<T>(a.inc, (start + t) * D + c);
            step_forward<double, D>(a, cur, nxt, x);
            __syncthreads();
            double* tmp = cur;
            cur = nxt;
            nxt = tmp;
        }

        // ---- G = upstream gradient
        const T* gsrc = static_cast<const T*>(a.grad_sig) + s * a.ld_grad;
        for (int64_t e = threadIdx.x; e < T_; e += blockDim.x) G[e] = (double)gsrc[e];
        __syncthreads();

        for (int64_t c = nseg - 1; c >= 0; --c) {
            const int64_t t0 = c * a.K;
            const int64_t t1 = min(len, t0 + (int64_t)a.K);
            // recompute the segment's states from its checkpoint
            for (int64_t e = threadIdx.x; e < T_; e += blockDim.x) states[e] = ckpt[c * T_ + e];
            __syncthreads();
            for (int64_t j = 0; j + 1 < t1 - t0; ++j) {
                U x[D];
#pragma unroll
                for (int q = 0; q < D; ++q) x[q] = (U)ld_inc<T>(a.inc, (start + t0 + j) * D + q);
                step_forward<U, D>(a, states + j * T_, states + (j + 1) * T_, x);
                __syncthreads();
            }
            // differentiate the steps of the segment in reverse
            for (int64_t j = t1 - t0 - 1; j >= 0; --j) {
                const int64_t t = t0 + j;
                const U* S = states + j * T_;
                U x[D];
#pragma unroll
                for (int q = 0; q < D; ++q) x[q] = (U)ld_inc<T>(a.inc, (start + t) * D + q);
                double gx[D];
#pragma unroll
                for (int q = 0; q < D; ++q) gx[q] = 0.0;

                for (int k = 1; k <= N; ++k) {
                    // chain values acc^{(k)}_i, i = 1..k-1 (prefix-chain formula)
                    for (int64_t e = a.db[1] + threadIdx.x; e < a.db[k]; e += blockDim.x) {
                        int i = 1;
                        while (e >= a.db[i + 1]) ++i;
                        const int64_t u = e - a.db[i];
                        U acc = U(1);
                        for (int m = 1; m <= i; ++m) {
                            const int64_t pref = u / a.pw[i - m];
                            acc = S[a.db[m] + pref] + acc * x[(int)(pref % D)] / U(k - m + 1);
                        }
                        chain[e] = acc;
                    }
                    __syncthreads();
                    // top of the chain: S'_k = S_k + acc_{k-1} (x) x
                    for (int64_t w = threadIdx.x; w < a.pw[k - 1]; w += blockDim.x) {
                        const double cw = (k == 1) ? 1.0 : (double)chain[a.db[k - 1] + w];
                        const double* gk = G + a.db[k] + w * D;
                        double sb = 0.0;
#pragma unroll
                        for (int q = 0; q < D; ++q) {
                            sb = fma(gk[q], (double)x[q], sb);
                            gx[q] = fma(gk[q], cw, gx[q]);
                        }
                        if (k >= 2) abar[a.db[k - 1] + w] = sb;
                    }
                    __syncthreads();
                    // down the chain: acc_i = S_i + acc_{i-1} (x) x / (k-i+1)
                    for (int i = k - 1; i >= 1; --i) {
                        const double inv = 1.0 / (double)(k - i + 1);
                        for (int64_t w = threadIdx.x; w < a.pw[i - 1]; w += blockDim.x) {
                            const double cw = (i == 1) ? 1.0 : (double)chain[a.db[i - 1] + w];
                            double* gi = G + a.db[i] + w * D;
                            const double* ai = abar + a.db[i] + w * D;
                            double sb = 0.0;
#pragma unroll
                            for (int q = 0; q < D; ++q) {
                                const double v = ai[q];
                                gi[q] += v;
                                sb = fma(v, (double)x[q], sb);
                                gx[q] = fma(v * inv, cw, gx[q]);
                            }
                            if (i >= 2) abar[a.db[i - 1] + w] = sb * inv;
                        }
                        __syncthreads();
                    }
                }
                // block reduction of dLoss/dx_t
#pragma unroll
                for (int q = 0; q < D; ++q) {
                    double v = gx[q];
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                    if (lane == 0) s_red[warp][q] = v;
                }
                __syncthreads();
                if (threadIdx.x < D) {
                    double v = 0.0;
                    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) v += s_red[w2][threadIdx.x];
                    static_cast<T*>(a.grad_inc)[(start + t) * D + threadIdx.x] = (T)v;
                }
                __syncthreads();
            }
        }
    }
}

// ------------------------------------------------------------------------
// Lane kernel

__host__ __device__ constexpr int64_t ipow_c(int64_t d, int e)
{
    return e <= 0 ? 1 : d * ipow_c(d, e - 1);
}

__host__ __device__ constexpr double inv_fact(int n)
{
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= (double)i;
    return 1.0 / f;
}

__host__ __device__ constexpr int64_t align16(int64_t b) { return (b + 15) / 16 * 16; }

template <typename T, int D, int N>
struct LaneLayout {
    static constexpr int P = N - 2;                      // path levels 1..N-2
    static constexpr int PP = P > 0 ? P : 1;
    static constexpr int64_t W = ipow_c(D, P > 0 ? P : 0);   // lanes per stream
    static constexpr int64_t NT = (W + 31) / 32 * 32;    // lane threads
    static constexpr int64_t NF = (1024 - NT) / 32 >= 4 ? 4 : (1024 - NT) / 32;  // fold warps
    static constexpr int64_t NTB = NT + 32 * NF;
    static constexpr int64_t NWARP = NT / 32;
    static constexpr int64_t TOPW = ipow_c(D, N);
    static constexpr bool GT_SMEM = TOPW * (int64_t)sizeof(T) <= 160 * 1024;
    static constexpr int CH = 32;                        // increment rows staged per chunk
    // ancestors: levels 1..P-1
    __host__ __device__ static constexpr int64_t anc_off(int k)
    {
        int64_t s = 0;
        for (int j = 1; j < k; ++j) s += ipow_c(D, j);
        return s;
    }
    __host__ __device__ static constexpr int64_t mbuf_off(int k)
    {
        int64_t s = 0;
        for (int j = 1; j < k; ++j) s += (int64_t)(N - j + 1) * ipow_c(D, j);
        return s;
    }
    static constexpr int64_t n_anc = anc_off(P > 1 ? P : 1);
    static constexpr int64_t n_mbuf = mbuf_off(P > 1 ? P : 1);
    static constexpr int64_t n_mlev = P >= 2 ? 3 * W : 0;
    // shared memory: per hand-off buffer b < NB the lane warps' gradient
    // partials, the fold warps' partials, the lanes' M vectors and the states
    // of shared prefixes; then fold-private ancestor data, the staged
    // increments, the top-level adjoints and the lanes' child adjoints G[pi m]
    // (kept here rather than in registers, which the fold warps cap)
    __host__ __device__ static constexpr int64_t per_buf()
    {
        return NWARP * 8 * 8 + NF * 8 * 8 + align16(n_mlev * 8) + align16(n_anc * 8);
    }
    __host__ __device__ static constexpr int64_t fixed()
    {
        return align16(D * W * 8) + align16(n_mbuf * 8) + align16(n_anc * 8) + align16((int64_t)CH * D * 8) +
               align16((int64_t)CH * D * (int64_t)sizeof(T)) +
               (GT_SMEM ? align16(TOPW * (int64_t)sizeof(T)) : 0);
    }
    static constexpr int NB = (4 * per_buf() + fixed() <= 200 * 1024) ? 4 : 2;   // hand-off buffers
    static constexpr int64_t o_gxw = 0;                                   // f64 [NB][NWARP][8]
    static constexpr int64_t o_anct = o_gxw + NB * NWARP * 8 * 8;         // f64 [NB][NF][8]
    static constexpr int64_t o_mlev = o_anct + NB * NF * 8 * 8;           // f64 [NB][3][W]
    static constexpr int64_t o_sanc = o_mlev + NB * align16(n_mlev * 8);  // f64 [NB][n_anc]
    static constexpr int64_t o_mbuf = o_sanc + NB * align16(n_anc * 8);
    static constexpr int64_t o_ganc = o_mbuf + align16(n_mbuf * 8);
    static constexpr int64_t o_xd = o_ganc + align16(n_anc * 8);          // f64 [CH][D]
    static constexpr int64_t o_xt = o_xd + align16((int64_t)CH * D * 8);  // T [CH][D]
    static constexpr int64_t o_gtop = o_xt + align16((int64_t)CH * D * (int64_t)sizeof(T));
    static constexpr int64_t o_gms = o_gtop + (GT_SMEM ? align16(TOPW * (int64_t)sizeof(T)) : 0);
    static constexpr int64_t bytes = o_gms + align16(D * W * 8);
    static constexpr int64_t mlev_stride = align16(n_mlev * 8) / 8;
    static constexpr int64_t sanc_stride = align16(n_anc * 8) / 8;
    // named barriers (0 is __syncthreads): lanes filled buffer b, fold warps
    // released buffer b, and among the fold warps
    __host__ __device__ static constexpr int bar_full(int b) { return 1 + b; }
    __host__ __device__ static constexpr int bar_empty(int b) { return 1 + NB + b; }
    static constexpr int bar_fold = 1 + 2 * NB;
    __host__ __device__ static constexpr int64_t db(int k) { return (ipow_c(D, k) - 1) / (D - 1); }
};

__device__ __forceinline__ void bar_sync_n(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void bar_arrive_n(int id, int n)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// One Chen step S <- S (x) exp(s x), s = -1 when NEG, of a lane's words at
// levels <= N-1: its path words sp[i-1] = S[pi_1..pi_i] and its children
// sm[m] = S[pi m].  xc[i] = x[pi_{i+1}].  Levels are updated from the top down
// so every chain reads pre-step values.
template <int D, int P, int PP, bool NEG>
__device__ __forceinline__ void lane_step(double (&sp)[PP], double (&sm)[D], const double (&x)[D],
                                          const double (&xc)[PP])
{
    constexpr double sg = NEG ? -1.0 : 1.0;
    double f0 = 1.0;  // F_0(pi): chain with divisors P+2-i
#pragma unroll
    for (int i = 1; i <= P; ++i) f0 = fma(f0, xc[i - 1] * (sg / (double)(P + 2 - i)), sp[i - 1]);
#pragma unroll
    for (int m = 0; m < D; ++m) sm[m] = fma(f0, sg * x[m], sm[m]);
#pragma unroll
    for (int i = P; i >= 1; --i) {
        double h = 1.0;  // F_0(pi_1..pi_{i-1}): divisors i+1-j
#pragma unroll
        for (int j = 1; j <= i - 1; ++j) h = fma(h, xc[j - 1] * (sg / (double)(i + 1 - j)), sp[j - 1]);
        sp[i - 1] = fma(h, sg * xc[i - 1], sp[i - 1]);
    }
}

// Sum of v[0..D) over the warp, scattered: returns the total of one letter in
// every lane whose low bits are zero (letter() tells which).  Halving steps
// exchange half of the remaining values per shuffle, so D values cost
// Q/2 + Q/4 + ... + (5 - log2 Q) shuffles instead of 5 D.
template <int D, typename V>
struct WarpScatter {
    static constexpr int Q = D > 4 ? 8 : (D > 2 ? 4 : 2);
    static constexpr int LQ = Q == 8 ? 3 : (Q == 4 ? 2 : 1);
    static __device__ __forceinline__ V run(const V (&v)[D], int lane)
    {
        V a[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) a[i] = (i < D) ? v[i] : V(0);
        int half = Q / 2;
#pragma unroll
        for (int st = 0; st < LQ; ++st) {
            const int off = 16 >> st;
            const bool up = (lane & off) != 0;
#pragma unroll
            for (int i = 0; i < Q / 2; ++i) {
                if (i < half) {
                    const V keep = up ? a[half + i] : a[i];
                    const V send = up ? a[i] : a[half + i];
                    a[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
                }
            }
            half >>= 1;
        }
        V r = a[0];
#pragma unroll
        for (int off = 16 >> LQ; off > 0; off >>= 1) r += __shfl_xor_sync(0xffffffffu, r, off);
        return r;
    }
    static __device__ __forceinline__ int letter(int lane)
    {
        int l = 0;
#pragma unroll
        for (int st = 0; st < LQ; ++st) l = 2 * l + ((lane >> (4 - st)) & 1);
        return l;
    }
    static __device__ __forceinline__ bool writer(int lane) { return (lane & ((16 >> (LQ - 1)) - 1)) == 0; }
};

// Fold warps, ancestor level K (1 <= K <= P-1): node u (strided over the
// fold threads) folds its children's M vectors into its own, updates its
// adjoint and adds its gradient term sum_q F_q(parent(u)) M_q(u) to letter
// u mod D.
template <typename T, int D, int N, int K>
__device__ __forceinline__ void fold_levels(int fl, const double* __restrict__ xr,
                                            const double* mlev, double* mbuf, double* ganc,
                                            const double* sanc, double (&gacc)[D])
{
    if constexpr (K >= 1) {
        using LY = LaneLayout<T, D, N>;
        constexpr int P = LY::P;
        constexpr int NQ = N - K + 1;
        constexpr int NU = (int)ipow_c(D, K);
        constexpr int64_t CS = ipow_c(D, K + 1);
        constexpr int NFT = (int)LY::NF * 32;
        const double* child = (K + 1 == P) ? mlev : (mbuf + LY::mbuf_off(K + 1));
#pragma unroll
        for (int u0 = 0; u0 < NU; u0 += NFT) {
            const int u = u0 + fl;
            if (u >= NU) break;
            double Mq[NQ];
            Mq[0] = ganc[LY::anc_off(K) + u];
#pragma unroll
            for (int q = 1; q < NQ; ++q) {
                double acc = 0.0;
#pragma unroll
                for (int cc = 0; cc < D; ++cc)
                    acc = fma(xr[cc], child[(q - 1) * CS + (int64_t)u * D + cc], acc);
                Mq[q] = acc;
            }
            if constexpr (K > 1) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) mbuf[LY::mbuf_off(K) + q * NU + u] = Mq[q];
            }
            double g = Mq[0];
#pragma unroll
            for (int q = 1; q < NQ; ++q) g = fma(Mq[q], inv_fact(q), g);
            ganc[LY::anc_off(K) + u] = g;
            // parent(u) = u / D at level K-1; the states of its prefixes are in sanc
            const int par = u / D;
            double contrib = 0.0;
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                double h = 1.0;
#pragma unroll
                for (int i = 1; i <= K - 1; ++i) {
                    const int pref = par / (int)ipow_c(D, K - 1 - i);
                    h = fma(h, xr[pref % D] * (1.0 / (double)(q + K + 1 - i)),
                            sanc[LY::anc_off(i) + pref]);
                }
                contrib = fma(h * inv_fact(q + 1), Mq[q], contrib);
            }
            const int l = u % D;
#pragma unroll
            for (int b = 0; b < D; ++b) gacc[b] += (b == l) ? contrib : 0.0;
        }
        bar_sync_n(LY::bar_fold, NFT);
        fold_levels<T, D, N, K - 1>(fl, xr, mlev, mbuf, ganc, sanc, gacc);
    }
}

template <typename T, int D, int N>
__global__ void __launch_bounds__(LaneLayout<T, D, N>::NTB, 1)
signature_backward_lanes(const BwdArgs a)
{
    using LY = LaneLayout<T, D, N>;
    constexpr int P = LY::P, PP = LY::PP, CH = LY::CH, NB = LY::NB;
    constexpr int W = (int)LY::W, NT = (int)LY::NT, NTB = (int)LY::NTB, NWARP = (int)LY::NWARP;
    constexpr bool GT_SMEM = LY::GT_SMEM;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* gxw = reinterpret_cast<double*>(smem_raw + LY::o_gxw);
    double* anct = reinterpret_cast<double*>(smem_raw + LY::o_anct);
    double* mlev = reinterpret_cast<double*>(smem_raw + LY::o_mlev);
    double* mbuf = reinterpret_cast<double*>(smem_raw + LY::o_mbuf);
    double* ganc = reinterpret_cast<double*>(smem_raw + LY::o_ganc);
    double* sanc = reinterpret_cast<double*>(smem_raw + LY::o_sanc);
    double* xd = reinterpret_cast<double*>(smem_raw + LY::o_xd);
    T* xt = reinterpret_cast<T*>(smem_raw + LY::o_xt);
    T* gtop_s = reinterpret_cast<T*>(smem_raw + LY::o_gtop);
    double* gms = reinterpret_cast<double*>(smem_raw + LY::o_gms);
    __shared__ int s_item;

    const int tid = (int)threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool fold = tid >= NT;               // the last warps fold ancestors and sum gradients
    const bool active = tid < W;
    const int pi = active ? tid : (W - 1);     // idle threads mirror the last lane, write nothing
    int c[PP];
    {
        int t = pi;
        c[0] = 0;
#pragma unroll
        for (int i = P - 1; i >= 0; --i) {
            c[i] = t % D;
            t /= D;
        }
    }
    // bit q: this lane publishes the state of its level-q prefix (it is the
    // first lane below that prefix)
    unsigned own = 0;
    {
        bool z = true;
#pragma unroll
        for (int q = P - 1; q >= 1; --q) {
            z = z && (c[q] == 0);
            if (z && active) own |= 1u << q;
        }
    }
    const int K = a.K;
    double* ck = reinterpret_cast<double*>(a.scratch + (int64_t)blockIdx.x * a.slot_bytes);
    constexpr int CKW = PP + D;   // words per lane per checkpoint

    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(a.queue, 1);
        __syncthreads();
        const int64_t s = s_item;
        if (s >= a.n_streams) break;
        const int64_t start = a.offsets[s];
        const int64_t len = a.offsets[s + 1] - start;
        const T* __restrict__ xs = static_cast<const T*>(a.inc) + start * D;
        T* __restrict__ gout = static_cast<T*>(a.grad_inc) + start * D;
        if ((len + K - 1) / K > a.max_segments) {
            for (int64_t e = tid; e < len * D; e += NTB) gout[e] = (T)NAN;
            continue;
        }
        const T* __restrict__ gsig = static_cast<const T*>(a.grad_sig) + s * a.ld_grad;

        // ---- forward pass over levels <= N-1, checkpoints every K steps
        double sp[PP], sm[D];
#pragma unroll
        for (int i = 0; i < PP; ++i) sp[i] = 0.0;
#pragma unroll
        for (int m = 0; m < D; ++m) sm[m] = 0.0;
        int kc = 0;
        int64_t seg = 0;
        for (int64_t t0 = 0; t0 < len; t0 += CH) {
            const int n = (int)min((int64_t)CH, len - t0);
            __syncthreads();
            for (int i = tid; i < n * D; i += NTB) xd[i] = (double)xs[t0 * D + i];
            __syncthreads();
            if (!fold) {
                for (int j = 0; j < n; ++j) {
                    if (kc == 0 && active) {
                        double* row = ck + seg * CKW * W + pi;
#pragma unroll
                        for (int i = 0; i < PP; ++i) row[i * W] = sp[i];
#pragma unroll
                        for (int m = 0; m < D; ++m) row[(PP + m) * W] = sm[m];
                    }
                    if (kc == 0) ++seg;
                    if (++kc == K) kc = 0;
                    double x[D], xc[PP];
#pragma unroll
                    for (int b = 0; b < D; ++b) x[b] = xd[j * D + b];
#pragma unroll
                    for (int i = 0; i < PP; ++i) xc[i] = (i < P) ? xd[j * D + c[i]] : 0.0;
                    lane_step<D, P, PP, false>(sp, sm, x, xc);
                }
            }
        }

        // ---- adjoint state from the upstream gradient
        double gp = (double)gsig[LY::db(P > 0 ? P : 0) + pi];
        if (active) {
#pragma unroll
            for (int m = 0; m < D; ++m) gms[m * W + pi] = (double)gsig[LY::db(N - 1) + (int64_t)pi * D + m];
        }
        if constexpr (GT_SMEM) {
            for (int64_t i = tid; i < LY::TOPW; i += NTB) {
                const int64_t l = i / (D * D);
                const int64_t j = i - l * (D * D);
                gtop_s[j * W + l] = gsig[LY::db(N) + i];
            }
        }
        // ancestor words of levels 1..P-1 are contiguous in the tensor from word 1
        for (int64_t i = tid; i < LY::n_anc; i += NTB) ganc[i] = (double)gsig[1 + i];
        const T* gtop_g = gsig + LY::db(N);

        // ---- reverse pass
        int rc = (len > 0) ? (int)((len - 1) % K) : 0;
        for (int64_t t1 = len; t1 > 0; t1 -= CH) {
            const int64_t t0 = t1 > CH ? t1 - CH : 0;
            const int n = (int)(t1 - t0);
            __syncthreads();
            for (int i = tid; i < n * D; i += NTB) {
                const T v = xs[t0 * D + i];
                xt[i] = v;
                xd[i] = (double)v;
            }
            __syncthreads();
            if (!fold) {
                using WS = WarpScatter<D, T>;
                for (int i = 0; i < n; ++i) {
                    const int j = n - 1 - i;
                    const int64_t t = t0 + j;
                    const int bb = i % NB;
                    const double* row = xd + j * D;
                    const T* rowt = xt + j * D;
                    double x[D], xc[PP];
#pragma unroll
                    for (int b = 0; b < D; ++b) x[b] = row[b];
#pragma unroll
                    for (int q = 0; q < PP; ++q) xc[q] = (q < P) ? row[c[q]] : 0.0;
                    // S_{t+1} -> S_t by the inverse step, re-anchored on checkpoints
                    lane_step<D, P, PP, true>(sp, sm, x, xc);
                    if (rc == 0) {
                        const double* crow = ck + (t / K) * CKW * W + pi;
#pragma unroll
                        for (int q = 0; q < PP; ++q) sp[q] = crow[q * W];
#pragma unroll
                        for (int m = 0; m < D; ++m) sm[m] = crow[(PP + m) * W];
                        rc = K - 1;
                    } else {
                        --rc;
                    }
                    // buffer bb is free once the fold warps are done with step i - NB
                    if (i >= NB) bar_sync_n(LY::bar_empty(bb), NTB);

                    // states of shared prefixes (levels 1..P-2) for the fold warps
                    if constexpr (P >= 3) {
                        double* sa = sanc + bb * LY::sanc_stride;
#pragma unroll
                        for (int q = 1; q <= P - 2; ++q)
                            if (own & (1u << q)) sa[LY::anc_off(q) + pi / (int)ipow_c(D, P - q)] = sp[q - 1];
                    }

                    // chains C_r over the first P-1 path letters, r = P+1, P+2, P+3
                    double h1 = 1.0, h2 = 1.0, h3 = 1.0;
#pragma unroll
                    for (int q = 1; q <= P - 1; ++q) {
                        h1 = fma(h1, xc[q - 1] * (1.0 / (double)(P + 1 - q)), sp[q - 1]);
                        h2 = fma(h2, xc[q - 1] * (1.0 / (double)(P + 2 - q)), sp[q - 1]);
                        h3 = fma(h3, xc[q - 1] * (1.0 / (double)(P + 3 - q)), sp[q - 1]);
                    }
                    double F0pi = 1.0, hm = 1.0;   // F_0(pi); hm = 2 F_1(pi)
                    if constexpr (P >= 1) {
                        F0pi = fma(h2, xc[P - 1] * 0.5, sp[P - 1]);
                        hm = fma(h3, xc[P - 1] * (1.0 / 3.0), sp[P - 1]);
                    }
                    const double F1pi = 0.5 * hm;

                    // subtree of pi: children and (constant) top-level adjoints
                    T gx[D];
#pragma unroll
                    for (int b = 0; b < D; ++b) gx[b] = T(0);
                    double M1 = 0.0, M2 = 0.0;
#pragma unroll
                    for (int m = 0; m < D; ++m) {
                        T g[D];
#pragma unroll
                        for (int b = 0; b < D; ++b)
                            g[b] = GT_SMEM ? gtop_s[(m * D + b) * W + pi]
                                           : __ldg(gtop_g + ((int64_t)pi * D + m) * D + b);
                        T y = T(0);
#pragma unroll
                        for (int b = 0; b < D; ++b) y = fma(rowt[b], g[b], y);
                        const T f = (T)fma(hm, x[m] * 0.5, sm[m]);          // F_0(pi m)
#pragma unroll
                        for (int b = 0; b < D; ++b) gx[b] = fma(f, g[b], gx[b]);
                        const double yd = (double)y;                        // M_1(pi m)
                        const double gmv = gms[m * W + pi];
                        gx[m] += (T)fma(F0pi, gmv, F1pi * yd);
                        M1 = fma(x[m], gmv, M1);
                        M2 = fma(x[m], yd, M2);
                        if (active) gms[m * W + pi] = gmv + yd;
                    }
                    const double M0 = gp;
                    if constexpr (P >= 1) {
                        // the lane's word pi extends parent(pi): sum_q F_q(parent(pi)) M_q(pi)
                        const T v = (T)fma(h1, M0, fma(0.5 * h2, M1, (h3 * (1.0 / 6.0)) * M2));
#pragma unroll
                        for (int b = 0; b < D; ++b) gx[b] += (b == c[P - 1]) ? v : T(0);
                    }
                    if constexpr (P >= 2) {
                        if (active) {
                            double* ml = mlev + bb * LY::mlev_stride;
                            ml[pi] = M0;
                            ml[W + pi] = M1;
                            ml[2 * W + pi] = M2;
                        }
                    }
                    gp = fma(0.5, M2, M0 + M1);
                    if (!active) {
#pragma unroll
                        for (int b = 0; b < D; ++b) gx[b] = T(0);
                    }
                    {
                        const T r = WS::run(gx, lane);
                        const int l = WS::letter(lane);
                        if (WS::writer(lane) && l < D) gxw[(bb * NWARP + warp) * 8 + l] = (double)r;
                    }
                    bar_arrive_n(LY::bar_full(bb), NTB);
                }
                // take the fold warps' last releases so every barrier is balanced
                for (int i = (n > NB ? n - NB : 0); i < n; ++i) bar_sync_n(LY::bar_empty(i % NB), NTB);
            } else {
                using WS = WarpScatter<D, double>;
                constexpr int NF = (int)LY::NF;
                const int fl = tid - NT;          // 0 .. 32 NF - 1
                const int fw = fl >> 5;
                for (int i = 0; i < n; ++i) {
                    const int j = n - 1 - i;
                    const int64_t t = t0 + j;
                    const int bb = i % NB;
                    bar_sync_n(LY::bar_full(bb), NTB);
                    double gacc[D];
#pragma unroll
                    for (int b = 0; b < D; ++b) gacc[b] = 0.0;
                    fold_levels<T, D, N, P - 1>(fl, xd + j * D, mlev + bb * LY::mlev_stride, mbuf,
                                                ganc, sanc + bb * LY::sanc_stride, gacc);
                    const double r = WS::run(gacc, lane);
                    const int l = WS::letter(lane);
                    if (WS::writer(lane) && l < D) anct[(bb * NF + fw) * 8 + l] = r;
                    bar_sync_n(LY::bar_fold, NF * 32);
                    if (fl < D) {
                        double v = 0.0;
#pragma unroll
                        for (int f2 = 0; f2 < NF; ++f2) v += anct[(bb * NF + f2) * 8 + fl];
#pragma unroll
                        for (int w2 = 0; w2 < NWARP; ++w2) v += gxw[(bb * NWARP + w2) * 8 + fl];
                        gout[t * D + fl] = (T)v;
                    }
                    bar_arrive_n(LY::bar_empty(bb), NTB);
                }
            }
        }
    }
}

// RPYB_BWD_BLOCK=1 routes every shape to the block kernel
bool lane_kernel_disabled()
{
    static const bool off = [] {
        const char* e = getenv("RPYB_BWD_BLOCK");
        return e && e[0] == '1';
    }();
    return off;
}

struct LaneEntry {
    void (*fn)(BwdArgs) = nullptr;
    int64_t smem = 0;
    int threads = 0;
    int64_t lanes = 0;
    int ckw = 0;
};

template <typename T, int D, int N>
bool lane_fill(LaneEntry& e)
{
    if constexpr (N >= 2 && ipow_c(D, N - 2) <= 992) {
        using LY = LaneLayout<T, D, N>;
        if constexpr (LY::bytes <= 200 * 1024) {
            e.fn = &signature_backward_lanes<T, D, N>;
            e.smem = LY::bytes;
            e.threads = (int)LY::NTB;
            e.lanes = LY::W;
            e.ckw = LY::PP + D;
            return true;
        }
    }
    return false;
}

template <typename T, int D>
bool lane_pick_d(int n, LaneEntry& e)
{
    switch (n) {
        case 2: return lane_fill<T, D, 2>(e);
        case 3: return lane_fill<T, D, 3>(e);
        case 4: return lane_fill<T, D, 4>(e);
        case 5: return lane_fill<T, D, 5>(e);
        case 6: return lane_fill<T, D, 6>(e);
        case 7: return lane_fill<T, D, 7>(e);
        case 8: return lane_fill<T, D, 8>(e);
        case 9: return lane_fill<T, D, 9>(e);
        case 10: return lane_fill<T, D, 10>(e);
        case 11: return lane_fill<T, D, 11>(e);
        default: return false;
    }
}

template <typename T>
bool lane_pick(int d, int n, LaneEntry& e)
{
    switch (d) {
        case 2: return lane_pick_d<T, 2>(n, e);
        case 3: return lane_pick_d<T, 3>(n, e);
        case 4: return lane_pick_d<T, 4>(n, e);
        case 5: return lane_pick_d<T, 5>(n, e);
        case 6: return lane_pick_d<T, 6>(n, e);
        case 7: return lane_pick_d<T, 7>(n, e);
        case 8: return lane_pick_d<T, 8>(n, e);
        default: return false;
    }
}

bool lane_entry(int mode, int d, int n, LaneEntry& e)
{
    if (lane_kernel_disabled()) return false;
    return mode == RPYB_F64 ? lane_pick<double>(d, n, e) : lane_pick<float>(d, n, e);
}

int64_t lane_slot_bytes(const LaneEntry& e, int64_t max_segments)
{
    return (max_segments * e.ckw * e.lanes * 8 + 255) / 256 * 256;
}

// blocks in flight for the lane kernel (one workspace slot each)
int64_t lane_slots(const LaneEntry& e, int64_t n_streams)
{
    int dev = 0, sms = 148, occ = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)e.smem) == cudaSuccess)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, e.fn, e.threads, (size_t)e.smem);
        cudaGetLastError();
    }
    return std::min<int64_t>(std::max<int64_t>(1, n_streams), (int64_t)sms * std::max(occ, 1));
}

template <typename T>
using BwdKernel = void (*)(BwdArgs);

template <typename T>
BwdKernel<T> pick(int d)
{
    switch (d) {
        case 1: return &signature_backward_kernel<T, 1>;
        case 2: return &signature_backward_kernel<T, 2>;
        case 3: return &signature_backward_kernel<T, 3>;
        case 4: return &signature_backward_kernel<T, 4>;
        case 5: return &signature_backward_kernel<T, 5>;
        case 6: return &signature_backward_kernel<T, 6>;
        case 7: return &signature_backward_kernel<T, 7>;
        case 8: return &signature_backward_kernel<T, 8>;
        default: return nullptr;
    }
}

int64_t slot_bytes_for(int mode, const Geometry& g, int K, int64_t max_segments)
{
    const int64_t T = g.size();
    const int64_t es = (mode == RPYB_F64) ? 8 : 4;
    int64_t b = 4 * T * 8 + T * es + (int64_t)K * T * es + max_segments * T * es;
    return (b + 255) / 256 * 256;
}

int backward_slots()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 2;
}

// Longest and shortest stream of a batch: out[0] = max length, out[1] =
// min length (both start at 0 and LLONG_MAX), by atomics over a grid-stride
// pass through the offsets.
__global__ void stream_length_range_kernel(const int64_t* __restrict__ offsets, int64_t n,
                                           long long* out)
{
    long long hi = 0, lo = LLONG_MAX;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const long long len = (long long)(offsets[i + 1] - offsets[i]);
        hi = len > hi ? len : hi;
        lo = len < lo ? len : lo;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const long long h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        const long long l2 = __shfl_xor_sync(0xffffffffu, lo, o);
        hi = h2 > hi ? h2 : hi;
        lo = l2 < lo ? l2 : lo;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, hi);
        atomicMin(out + 1, lo);
    }
}

// Reads the longest and shortest stream length of the batch into the host
// values (one small kernel and a 16-byte read that waits for stream s).
int stream_length_range(const int64_t* offsets, int64_t n, void* scratch16, cudaStream_t s,
                        int64_t* max_len, int64_t* min_len)
{
    long long init[2] = {0, LLONG_MAX};
    long long got[2] = {0, 0};
    long long* d = static_cast<long long*>(scratch16);
    RPYB_CUDA(cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int threads = 256;
    const int64_t blocks = std::min<int64_t>((n + threads - 1) / threads, 1024);
    stream_length_range_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), threads, 0, s>>>(offsets,
                                                                                         n, d);
    RPYB_CUDA(cudaGetLastError());
    RPYB_CUDA(cudaMemcpyAsync(got, d, sizeof(got), cudaMemcpyDeviceToHost, s));
    RPYB_CUDA(cudaStreamSynchronize(s));
    *max_len = got[0];
    *min_len = got[1];
    return RPYB_OK;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_signature_backward_workspace_size(int mode, int32_t width, int32_t depth,
                                                        int64_t n_streams, int64_t max_len,
                                                        int32_t checkpoint_every)
{
    Geometry g;
    if ((mode != RPYB_F32 && mode != RPYB_F64) || make_geometry(width, depth, g)) return -1;
    if (checkpoint_every < 1 || max_len < 0 || n_streams < 0) return -1;
    const int64_t segs = std::max<int64_t>(1, (max_len + checkpoint_every - 1) / checkpoint_every);
    LaneEntry e;
    if (lane_entry(mode, width, depth, e))
        return 256 + lane_slots(e, n_streams) * lane_slot_bytes(e, segs);
    const int64_t slots = std::min<int64_t>(backward_slots(), std::max<int64_t>(1, n_streams));
    return 256 + slots * slot_bytes_for(mode, g, checkpoint_every, segs);
}

RPYB_API int rpyb_signature_backward(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                     const int64_t* offsets, int64_t max_len,
                                     const void* increments, const void* grad_sig,
                                     int64_t ld_grad, void* grad_inc, int32_t checkpoint_every,
                                     void* workspace, size_t workspace_bytes, void* stream)
{
    int rc;
    if (mode != RPYB_F32 && mode != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported mode");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (width > 8) return fail(RPYB_E_UNSUPPORTED, "signature backward supports width <= 8");
    if (depth < 1) return fail(RPYB_E_INVALID, "signature backward needs depth >= 1");
    if (n_streams < 0 || max_len < -1) return fail(RPYB_E_INVALID, "negative size");
    if (checkpoint_every < 1) return fail(RPYB_E_INVALID, "checkpoint interval must be >= 1");
    if (n_streams == 0) return RPYB_OK;
    if (!offsets || !grad_sig || !grad_inc) return fail(RPYB_E_INVALID, "null pointer");
    if (ld_grad != 0 && ld_grad < g.size()) return fail(RPYB_E_INVALID, "ld_grad too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Validate the caller's bound before sizing anything from it: the
    // checkpoint scratch of every stream is sized by max_len.
    int64_t longest = 0, shortest = 0;
    {
        // 16 bytes of scratch: the head of the caller's workspace when there
        // is one (rewritten below once the check has completed)
        Scratch probe(workspace_bytes >= 16 ? workspace : nullptr, workspace_bytes, s);
        void* p16 = nullptr;
        if ((rc = probe.get(16, &p16))) return rc;
        if ((rc = stream_length_range(offsets, n_streams, p16, s, &longest, &shortest))) return rc;
    }
    if (shortest < 0) return fail(RPYB_E_INVALID, "offsets must be non-decreasing");
    if (max_len == -1) {
        max_len = longest;
    } else if (longest > max_len) {
        return fail(RPYB_E_INVALID, "a stream has " + std::to_string(longest) +
                                        " increments, more than max_len = " +
                                        std::to_string(max_len));
    }
    const int64_t need = rpyb_signature_backward_workspace_size(mode, width, depth, n_streams,
                                                                max_len, checkpoint_every);
    Scratch scratch(workspace, workspace_bytes, s);
    void* ws = nullptr;
    if ((rc = scratch.get((size_t)need, &ws))) return rc;

    BwdArgs a{};
    a.width = width;
    a.depth = depth;
    a.n_streams = n_streams;
    a.offsets = offsets;
    a.inc = increments;
    a.grad_sig = grad_sig;
    a.ld_grad = ld_grad;
    a.grad_inc = grad_inc;
    a.K = checkpoint_every;
    a.max_segments = std::max<int64_t>(1, (max_len + checkpoint_every - 1) / checkpoint_every);
    a.T = g.size();
    for (int k = 0; k <= kMaxDepth + 1; ++k) a.db[k] = g.db[k];
    for (int k = 0; k <= kMaxDepth; ++k) a.pw[k] = g.pw[k];
    a.queue = static_cast<int*>(ws);
    a.scratch = static_cast<char*>(ws) + 256;
    RPYB_CUDA(cudaMemsetAsync(ws, 0, sizeof(int), s));
    LaneEntry e;
    if (lane_entry(mode, width, depth, e)) {
        a.slot_bytes = lane_slot_bytes(e, a.max_segments);
        const int64_t slots = lane_slots(e, n_streams);
        e.fn<<<(unsigned)slots, e.threads, (size_t)e.smem, s>>>(a);
        RPYB_CUDA(cudaGetLastError());
        return RPYB_OK;
    }
    a.slot_bytes = slot_bytes_for(mode, g, checkpoint_every, a.max_segments);
    const int64_t slots = std::min<int64_t>(backward_slots(), n_streams);
    if (mode == RPYB_F64) {
        auto fn = pick<double>(width);
        fn<<<(unsigned)slots, kBwdThreads, 0, s>>>(a);
    } else {
        auto fn = pick<float>(width);
        fn<<<(unsigned)slots, kBwdThreads, 0, s>>>(a);
    }
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

}  // extern "C"
