// Reverse-mode derivative of batched signatures (the signature adjoint).
//
// For S_{t+1} = S_t (x) exp(x_t) and an upstream gradient G_L = dLoss/dS_L
// (e.g. W for Loss = <W, S_L>), one block walks a stream backwards:
//
//   * checkpoint pass: S_t is propagated forwards in float64 and stored every
//     K steps (the only states kept);
//   * per segment (last first): the K states of the segment are recomputed
//     from its checkpoint, then for t = segment end .. segment start the step
//     S_{t+1} = S_t (x) exp(x_t) is differentiated through its Horner chains
//       acc_1 = S_1 + x/k, acc_i = S_i + acc_{i-1} (x) x/(k-i+1),
//       S'_k  = S_k + acc_{k-1} (x) x,
//     giving dLoss/dx_t and G_t = dLoss/dS_t from G_{t+1} (the reverse Chen
//     product, i.e. the adjoint of right multiplication by exp(x_t)).
//
// The reference has no reverse-mode derivative (its sig_derivative is
// forward mode, algebra/src/lite_context.h:577-636); results are checked
// against float64 central finite differences and that forward derivative.
//
// Precision: the gradient accumulator G is float64 in both modes; mode
// RPYB_F32 recomputes states and chains in float32 from float32 checkpoints
// (written from the float64 checkpoint pass), RPYB_F64 does everything in
// float64.  Per-block scratch lives in the workspace.
#include <algorithm>

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
            // the caller's max_len does not bound this stream: no scratch for
            // its checkpoints, so its gradient is reported as NaN
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
    if (n_streams < 0 || max_len < 0) return fail(RPYB_E_INVALID, "negative size");
    if (checkpoint_every < 1) return fail(RPYB_E_INVALID, "checkpoint interval must be >= 1");
    if (n_streams == 0) return RPYB_OK;
    if (!offsets || !grad_sig || !grad_inc) return fail(RPYB_E_INVALID, "null pointer");
    if (ld_grad != 0 && ld_grad < g.size()) return fail(RPYB_E_INVALID, "ld_grad too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
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
    a.slot_bytes = slot_bytes_for(mode, g, checkpoint_every, a.max_segments);
    const int64_t slots = std::min<int64_t>(backward_slots(), n_streams);
    RPYB_CUDA(cudaMemsetAsync(ws, 0, sizeof(int), s));
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
