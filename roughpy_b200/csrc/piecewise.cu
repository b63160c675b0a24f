// Queries against a piecewise abelian stream: a sequence of (interval, Lie
// element) pieces (RoughPy's PiecewiseAbelianStream).
//
// Reference path (streams/src/stream.cpp:54-171 with
// streams/src/stream_base.cpp:81-96 and
// streams/src/piecewise_abelian_stream.cpp:154-189): the query is trimmed
// to the support and dissected into maximal dyadic intervals; for each dyadic
// interval [a, b) the pieces are scanned in order until one starts at or
// after b, and every piece that meets [a, b) contributes its Lie element,
// whole when it lies inside [a, b) and otherwise scaled by
// (piece.sup - a) / (piece.sup - piece.inf) (the reference's second branch
// tests `pb <= pb`, so every partial overlap takes this multiplier; that is
// reproduced here).  The contributions of one dyadic interval are combined by
// CBH, and the dyadic results by CBH again; the signature is
// exp(l2t(log-signature)).
//
// By associativity of the product of exponentials, the nested CBHs equal the
// log of the ordered product of exp(l2t(m_i L_i)) over every (dyadic
// interval, piece) pair of the query.  On the device: scale the piece rows,
// map them to tensors and exponentiate (batched over all pairs of all
// queries), multiply each query's factors in order (one gathered product per
// position), then take the float64 log and the Lie projection.
#include <algorithm>
#include <cmath>
#include <vector>

#include "stream_ops.cuh"

namespace rpyb {
namespace {

// out[i] <- mult[i] * lies[piece[i]]  (rows of L values)
__global__ void scaled_rows_kernel(double* __restrict__ out, const double* __restrict__ lies,
                                   int64_t ld_lies, const int64_t* __restrict__ piece,
                                   const double* __restrict__ mult, int64_t L, int64_t n)
{
    const int64_t total = n * L;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / L, c = e - i * L;
        out[e] = mult[i] * lies[piece[i] * ld_lies + c];
    }
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int rpyb_piecewise_query(int32_t width, int32_t depth, int64_t n_pieces,
                                  const double* piece_inf, const double* piece_sup,
                                  const double* piece_lies, int64_t ld_lies, double support_inf,
                                  double support_sup, int32_t default_resolution,
                                  int64_t n_queries, const double* inf_host,
                                  const double* sup_host, int32_t resolution, double* out_logsig,
                                  int64_t ld_logsig, double* out_sig, int64_t ld_sig, void* stream)
{
    int rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n_pieces < 0 || n_queries < 0) return fail(RPYB_E_INVALID, "negative size");
    if (n_queries == 0) return RPYB_OK;
    if (!inf_host || !sup_host) return fail(RPYB_E_INVALID, "null interval arrays");
    if (n_pieces > 0 && (!piece_inf || !piece_sup || !piece_lies))
        return fail(RPYB_E_INVALID, "null piece arrays");
    if (!out_logsig && !out_sig) return fail(RPYB_E_INVALID, "no output requested");
    if (default_resolution < -60 || default_resolution > 60)
        return fail(RPYB_E_INVALID, "resolution out of range");
    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;
    const int64_t T = g.size(), L = maps->lie_dim;
    if (n_pieces > 0 && ld_lies < L) return fail(RPYB_E_INVALID, "ld_lies too small");
    if (out_logsig && ld_logsig < L) return fail(RPYB_E_INVALID, "ld_logsig too small");
    if (out_sig && ld_sig < T) return fail(RPYB_E_INVALID, "ld_sig too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    std::vector<int64_t> k, poff;
    std::vector<int32_t> p;
    if ((rc = refine_and_dissect(n_queries, inf_host, sup_host, support_inf, support_sup,
                                 default_resolution, resolution, k, p, poff)))
        return rc;

    // (piece, multiplier) factors of every query, in order
    std::vector<int64_t> fpiece, qoff(n_queries + 1, 0);
    std::vector<double> fmult;
    for (int64_t q = 0; q < n_queries; ++q) {
        for (int64_t i = poff[q]; i < poff[q + 1]; ++i) {
            const double a = std::ldexp((double)k[i], -p[i]);
            const double b = std::ldexp((double)(k[i] + 1), -p[i]);
            for (int64_t j = 0; j < n_pieces; ++j) {
                const double pa = piece_inf[j], pb = piece_sup[j];
                if (pa >= b) break;
                if (pb <= a) continue;
                double mult = 1.0;
                if (!(pa >= a && pb <= b)) mult = (pb - a) / (pb - pa);
                fpiece.push_back(j);
                fmult.push_back(mult);
            }
        }
        qoff[q + 1] = (int64_t)fpiece.size();
    }

    // device, in chunks of queries whose factors fit a memory budget
    const int64_t max_rows = std::max<int64_t>(1, ((int64_t)1 << 30) / (T * 8));
    std::vector<int64_t> starts{0};
    for (int64_t q = 0; q < n_queries; ++q) {
        const int64_t q0 = starts.back();
        const bool too_many = (q - q0) >= max_rows ||
                              (q > q0 && qoff[q + 1] - qoff[q0] > max_rows);
        if (too_many) starts.push_back(q);
    }
    starts.push_back(n_queries);
    int64_t max_q = 0, max_f = 0;
    for (size_t c = 0; c + 1 < starts.size(); ++c) {
        max_q = std::max(max_q, starts[c + 1] - starts[c]);
        max_f = std::max(max_f, qoff[starts[c + 1]] - qoff[starts[c]]);
    }
    const size_t acc_b = (size_t)((max_q * T * 8 + 255) / 256 * 256);
    const size_t fin_b = finish_scratch_bytes(g, L, max_q);
    const size_t rows_b = (size_t)((std::max<int64_t>(max_f, 1) * T * 8 + 255) / 256 * 256);
    const size_t lrows_b = (size_t)((std::max<int64_t>(max_f, 1) * L * 8 + 255) / 256 * 256);
    const size_t meta_b = (size_t)((std::max<int64_t>(max_f, 1) * 16 + 255) / 256 * 256);
    const int64_t exp_ws = rpyb_ft_exp_workspace_size(RPYB_F64, width, depth,
                                                      std::max<int64_t>(max_f, 1));
    if (exp_ws < 0) return (int)exp_ws;
    const size_t exp_b = (size_t)std::max<int64_t>(exp_ws, 1);
    Scratch sc(nullptr, 0, s);
    void* mem = nullptr;
    if ((rc = sc.get(acc_b + fin_b + 2 * rows_b + lrows_b + meta_b + exp_b, &mem))) return rc;
    char* base = static_cast<char*>(mem);
    double* acc = reinterpret_cast<double*>(base);
    void* fin_mem = base + acc_b;
    double* emb = reinterpret_cast<double*>(base + acc_b + fin_b);
    double* ex = reinterpret_cast<double*>(base + acc_b + fin_b + rows_b);
    double* lrows = reinterpret_cast<double*>(base + acc_b + fin_b + 2 * rows_b);
    int64_t* d_piece = reinterpret_cast<int64_t*>(base + acc_b + fin_b + 2 * rows_b + lrows_b);
    double* d_mult = reinterpret_cast<double*>(d_piece + std::max<int64_t>(max_f, 1));
    void* exp_mem = base + acc_b + fin_b + 2 * rows_b + lrows_b + meta_b;

    for (size_t c = 0; c + 1 < starts.size(); ++c) {
        const int64_t q0 = starts[c], q1 = starts[c + 1], m = q1 - q0;
        const int64_t f0 = qoff[q0], nf = qoff[q1] - f0;
        const bool chain = chain_products_available(g) && nf > 0;
        if (!chain && (rc = unit_rows(RPYB_F64, acc, T, T, nullptr, m, s))) return rc;
        if (nf > 0) {
            RPYB_CUDA(cudaMemcpyAsync(d_piece, fpiece.data() + f0, (size_t)nf * 8,
                                      cudaMemcpyHostToDevice, s));
            RPYB_CUDA(cudaMemcpyAsync(d_mult, fmult.data() + f0, (size_t)nf * 8,
                                      cudaMemcpyHostToDevice, s));
            const unsigned blocks =
                (unsigned)std::max<int64_t>(1, std::min<int64_t>((nf * L + 255) / 256, 148 * 16));
            scaled_rows_kernel<<<blocks, 256, 0, s>>>(lrows, piece_lies, ld_lies, d_piece, d_mult, L,
                                                      nf);
            RPYB_CUDA(cudaGetLastError());
            // the sparse map accumulates: clear its output first
            RPYB_CUDA(cudaMemsetAsync(emb, 0, (size_t)(nf * T * 8), s));
            if ((rc = rpyb_sparse_map(RPYB_F64, T, L, nf, maps->l2t_ptr, maps->l2t_idx,
                                      maps->l2t_val, emb, lrows, T, L, 1.0, s)) ||
                (rc = rpyb_ft_exp(RPYB_F64, width, depth, nf, ex, emb, T, T, -1, exp_mem, exp_b,
                                  s)))
                return rc;
            std::vector<int64_t> loff(m + 1), rows(nf);
            for (int64_t i = 0; i <= m; ++i) loff[i] = qoff[q0 + i] - f0;
            for (int64_t i = 0; i < nf; ++i) rows[i] = i;
            if (chain && chain_lie_available(g, *maps)) {
                // products, log and Hall projection in one kernel
                double* lsq = out_logsig ? out_logsig + q0 * ld_logsig : nullptr;
                int64_t ld_lie = 0;
                double* lie = finish_lie_rows(g, L, m, fin_mem, lsq, ld_logsig, &ld_lie);
                if ((rc = chain_products_lie(RPYB_F64, g, m, ex, loff, rows, *maps, lie, ld_lie,
                                             s)) ||
                    (rc = finish_queries(g, *maps, m, acc, true, lsq, ld_logsig,
                                         out_sig ? out_sig + q0 * ld_sig : nullptr, ld_sig,
                                         fin_mem, fin_b, s, true)))
                    return rc;
                continue;
            }
            if ((rc = chain ? chain_products(RPYB_F64, g, m, acc, ex, loff, rows, true, s)
                            : ordered_products(RPYB_F64, RPYB_F64, g, m, acc, ex, loff, rows, s)))
                return rc;
        }
        if ((rc = finish_queries(g, *maps, m, acc, chain,
                                 out_logsig ? out_logsig + q0 * ld_logsig : nullptr,
                                 ld_logsig, out_sig ? out_sig + q0 * ld_sig : nullptr, ld_sig,
                                 fin_mem, fin_b, s)))
            return rc;
    }
    return RPYB_OK;
}

}  // extern "C"
