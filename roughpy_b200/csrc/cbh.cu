// Batched Campbell-Baker-Hausdorff products of Lie elements:
//   out[q] = t2l(log(exp(l2t(x_0)) exp(l2t(x_1)) ...))   over list q's items,
// the quantity Context::cbh returns for one list (algebra/src/context.cpp:187-208:
// an fmexp chain from the unit over the non-zero elements, then log and the
// tensor->Lie map).  Here all lists of a batch are done together: one
// sparse map and one exp over every item, the fused chain-product kernel with
// its float64 log (one block per list), and one Hall projection; all in
// float64.  A list of one element returns it unchanged, as the reference
// does; an empty list gives zero.
#include <algorithm>
#include <vector>

#include "stream_ops.cuh"

namespace rpyb {
namespace {

__global__ void copy_lie_rows_kernel(double* __restrict__ out, int64_t ld_out,
                                     const double* __restrict__ in, int64_t ld_in,
                                     const int64_t* __restrict__ dst, const int64_t* __restrict__ src,
                                     int64_t n, int64_t L)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * L;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / L, c = e - r * L;
        out[dst[r] * ld_out + c] = in[src[r] * ld_in + c];
    }
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int rpyb_cbh(int32_t width, int32_t depth, int64_t n_lists, const int64_t* offsets_host,
                      const double* lies, int64_t ld_lies, double* out, int64_t ld_out,
                      void* stream)
{
    int rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n_lists < 0) return fail(RPYB_E_INVALID, "negative number of lists");
    if (n_lists == 0) return RPYB_OK;
    if (!offsets_host || !out) return fail(RPYB_E_INVALID, "null pointer");
    if (offsets_host[0] != 0) return fail(RPYB_E_INVALID, "offsets must start at 0");
    for (int64_t q = 0; q < n_lists; ++q)
        if (offsets_host[q + 1] < offsets_host[q])
            return fail(RPYB_E_INVALID, "offsets must be non-decreasing");
    const int64_t n_items = offsets_host[n_lists];
    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;
    const int64_t T = g.size(), L = maps->lie_dim;
    if (n_items > 0 && (!lies || ld_lies < L)) return fail(RPYB_E_INVALID, "bad Lie rows");
    if (ld_out < L) return fail(RPYB_E_INVALID, "ld_out too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // chunks of lists whose items fit a memory budget of tensor rows
    const int64_t max_rows = std::max<int64_t>(1, ((int64_t)1 << 30) / (T * 8));
    std::vector<int64_t> starts{0};
    for (int64_t q = 0; q < n_lists; ++q) {
        const int64_t q0 = starts.back();
        if (q > q0 && ((q - q0) >= max_rows || offsets_host[q + 1] - offsets_host[q0] > max_rows))
            starts.push_back(q);
    }
    starts.push_back(n_lists);
    int64_t max_q = 0, max_f = 1;
    for (size_t c = 0; c + 1 < starts.size(); ++c) {
        max_q = std::max(max_q, starts[c + 1] - starts[c]);
        max_f = std::max(max_f, offsets_host[starts[c + 1]] - offsets_host[starts[c]]);
    }
    auto up = [](int64_t b) { return (size_t)((b + 255) / 256 * 256); };
    const size_t acc_b = up(max_q * T * 8);
    const size_t fin_b = finish_scratch_bytes(g, L, max_q);
    const size_t rows_b = up(max_f * T * 8);
    const int64_t exp_ws = rpyb_ft_exp_workspace_size(RPYB_F64, width, depth, max_f);
    if (exp_ws < 0) return (int)exp_ws;
    const size_t exp_b = (size_t)std::max<int64_t>(exp_ws, 1);
    // single-element lists: (destination list, source item) pairs
    std::vector<int64_t> single;
    for (int64_t q = 0; q < n_lists; ++q)
        if (offsets_host[q + 1] - offsets_host[q] == 1) single.push_back(q);
    const size_t single_b = up((int64_t)std::max<size_t>(single.size(), 1) * 16);
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    if ((rc = sc.get(acc_b + fin_b + 2 * rows_b + exp_b + single_b, &mem))) return rc;
    char* base = static_cast<char*>(mem);
    double* acc = reinterpret_cast<double*>(base);
    void* fin_mem = base + acc_b;
    double* emb = reinterpret_cast<double*>(base + acc_b + fin_b);
    double* ex = reinterpret_cast<double*>(base + acc_b + fin_b + rows_b);
    void* exp_mem = base + acc_b + fin_b + 2 * rows_b;
    int64_t* d_single = reinterpret_cast<int64_t*>(base + acc_b + fin_b + 2 * rows_b + exp_b);

    for (size_t c = 0; c + 1 < starts.size(); ++c) {
        const int64_t q0 = starts[c], q1 = starts[c + 1], m = q1 - q0;
        const int64_t f0 = offsets_host[q0], nf = offsets_host[q1] - f0;
        const bool chain = chain_products_available(g) && nf > 0;
        if (!chain && (rc = unit_rows(RPYB_F64, acc, T, T, nullptr, m, s))) return rc;
        if (nf > 0) {
            // exp(l2t(x)) for every item of the chunk
            RPYB_CUDA(cudaMemsetAsync(emb, 0, (size_t)(nf * T * 8), s));
            if ((rc = rpyb_sparse_map(RPYB_F64, T, L, nf, maps->l2t_ptr, maps->l2t_idx,
                                      maps->l2t_val, emb, lies + f0 * ld_lies, T, ld_lies, 1.0,
                                      s)) ||
                (rc = rpyb_ft_exp(RPYB_F64, width, depth, nf, ex, emb, T, T, -1, exp_mem, exp_b,
                                  s)))
                return rc;
            std::vector<int64_t> loff(m + 1), rows(nf);
            for (int64_t i = 0; i <= m; ++i) loff[i] = offsets_host[q0 + i] - f0;
            for (int64_t i = 0; i < nf; ++i) rows[i] = i;
            if (chain && chain_lie_available(g, *maps)) {
                // products, log and Hall projection in one kernel
                if ((rc = chain_products_lie(RPYB_F64, g, m, ex, loff, rows, *maps,
                                             out + q0 * ld_out, ld_out, s)))
                    return rc;
                continue;
            }
            if ((rc = chain ? chain_products(RPYB_F64, g, m, acc, ex, loff, rows, true, s)
                            : ordered_products(RPYB_F64, RPYB_F64, g, m, acc, ex, loff, rows, s)))
                return rc;
        }
        if ((rc = finish_queries(g, *maps, m, acc, chain, out + q0 * ld_out, ld_out, nullptr, 0,
                                 fin_mem, fin_b, s)))
            return rc;
    }
    if (!single.empty()) {
        std::vector<int64_t> pairs(2 * single.size());
        for (size_t i = 0; i < single.size(); ++i) {
            pairs[i] = single[i];
            pairs[single.size() + i] = offsets_host[single[i]];
        }
        RPYB_CUDA(cudaMemcpyAsync(d_single, pairs.data(), pairs.size() * 8, cudaMemcpyHostToDevice,
                                  s));
        const int64_t n = (int64_t)single.size();
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n * L + 255) / 256,
                                                                                 4096));
        copy_lie_rows_kernel<<<blocks, 256, 0, s>>>(out, ld_out, lies, ld_lies, d_single,
                                                    d_single + n, n, L);
        RPYB_CUDA(cudaGetLastError());
        // the host pairs must outlive the asynchronous copy
        RPYB_CUDA(cudaStreamSynchronize(s));
    }
    return RPYB_OK;
}

}  // extern "C"
