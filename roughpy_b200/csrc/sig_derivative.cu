// Forward-mode derivative of signatures with respect to Lie perturbations
// (RoughPy's Context::sig_derivative), batched over independent lists.
//
// For a list of pairs (x_i, p_i) of Lie elements (the log-signature of an
// interval and its perturbation), the reference computes
// (algebra/src/lite_context.h:577-636, LiteContext::sig_derivative_impl)
//
//   result = 0;  for each i:  E_i = exp(X_i),  X_i = l2t(x_i),  P_i = l2t(p_i)
//     result <- result * E_i + E_i * sum_{k=0..depth} (-1)^k ad_{X_i}^k(P_i) / (k+1)!
//
// (derive_series_compute: ad_X(Y) = X Y - Y X).  The series term
// E * sum (...) is the derivative of exp at X in the direction P, so a list
// of one pair gives d/de exp(X + e P) exactly.  The recurrence is reproduced
// as the reference states it, for any list length.
//
// B200 layout: every item of every list is independent until the final
// recurrence, so the Lie embeddings, exponentials and commutator series run
// as batched product launches over all items at once ([items, T] rows); the
// per-list recurrence is then one gathered product launch per list position.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "product.cuh"
#include "stream_ops.cuh"

namespace rpyb {
namespace {

// y <- a x + b y over n rows of `cols` values (row strides ld)
template <typename T>
__global__ void axpby_kernel(T* __restrict__ y, const T* __restrict__ x, double a, double b,
                             int64_t cols, int64_t n, int64_t ld)
{
    const int64_t total = n * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / cols, c = e - i * cols;
        y[i * ld + c] = (T)(a * (double)x[i * ld + c] + b * (double)y[i * ld + c]);
    }
}

// out[q[i]] <- tmp[i] + add[item[i]]
template <typename T>
__global__ void scatter_add_kernel(T* __restrict__ out, int64_t ld_out, const T* __restrict__ tmp,
                                   const T* __restrict__ add, int64_t cols,
                                   const int64_t* __restrict__ q, const int64_t* __restrict__ item,
                                   int64_t n)
{
    const int64_t total = n * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / cols, c = e - i * cols;
        out[q[i] * ld_out + c] = tmp[i * cols + c] + add[item[i] * cols + c];
    }
}

unsigned grid_of(int64_t total)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
}

template <typename T>
int axpby(T* y, const T* x, double a, double b, int64_t cols, int64_t n, int64_t ld, cudaStream_t s)
{
    if (n <= 0) return RPYB_OK;
    axpby_kernel<T><<<grid_of(n * cols), 256, 0, s>>>(y, x, a, b, cols, n, ld);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

// out <- lhs (x) rhs over n contiguous rows (stride T)
int mul_rows(int dtype, const Geometry& g, int64_t n, void* out, const void* lhs, const void* rhs,
             cudaStream_t s)
{
    return rpyb_ft_mul_gather(dtype, g.width, g.depth, n, out, lhs, rhs, g.size(), nullptr,
                              nullptr, nullptr, 0, s);
}

template <typename T>
int derivative(const Geometry& g, int64_t n_lists, const int64_t* off, const T* logsig,
               const T* pert, int64_t ld_lie, T* out, int64_t ld_out, char* ws,
               const int64_t* d_ptr[2], const int64_t* d_idx[2], const double* d_val[2],
               int64_t lie_dim, cudaStream_t s)
{
    const int dtype = sizeof(T) == 8 ? RPYB_F64 : RPYB_F32;
    const int64_t T_ = g.size();
    const int64_t n = off[n_lists];
    const size_t rb = (size_t)((n * T_ * (int64_t)sizeof(T) + 255) / 256 * 256);
    T* X = reinterpret_cast<T*>(ws);
    T* E = reinterpret_cast<T*>(ws + rb);
    T* S = reinterpret_cast<T*>(ws + 2 * rb);
    T* A = reinterpret_cast<T*>(ws + 3 * rb);
    T* U = reinterpret_cast<T*>(ws + 4 * rb);
    T* V = reinterpret_cast<T*>(ws + 5 * rb);
    char* rest = ws + 6 * rb;
    const size_t exp_ws = (size_t)std::max<int64_t>(
        1, rpyb_ft_exp_workspace_size(dtype, g.width, g.depth, std::max<int64_t>(n, 1)));
    char* exp_scratch = rest;
    rest += (exp_ws + 255) / 256 * 256;
    int rc;
    // the sparse map accumulates: clear its outputs first
    RPYB_CUDA(cudaMemsetAsync(X, 0, (size_t)(n * T_ * sizeof(T)), s));
    RPYB_CUDA(cudaMemsetAsync(S, 0, (size_t)(n * T_ * sizeof(T)), s));
    if ((rc = rpyb_sparse_map(dtype, T_, lie_dim, n, d_ptr[0], d_idx[0], d_val[0], X, logsig, T_,
                              ld_lie, 1.0, s)) ||
        (rc = rpyb_sparse_map(dtype, T_, lie_dim, n, d_ptr[0], d_idx[0], d_val[0], S, pert, T_,
                              ld_lie, 1.0, s)))
        return rc;
    if ((rc = rpyb_ft_exp(dtype, g.width, g.depth, n, E, X, T_, T_, -1, exp_scratch, exp_ws, s)))
        return rc;
    // series S = P - [X,P]/2! + [X,[X,P]]/3! - ...; A holds ad_X^k(P)
    RPYB_CUDA(cudaMemcpyAsync(A, S, (size_t)(n * T_ * sizeof(T)), cudaMemcpyDeviceToDevice, s));
    double factor = 1.0;
    for (int k = 1; k <= g.depth; ++k) {
        // A <- X A - A X
        if ((rc = mul_rows(dtype, g, n, U, X, A, s)) || (rc = mul_rows(dtype, g, n, V, A, X, s)))
            return rc;
        RPYB_CUDA(cudaMemcpyAsync(A, U, (size_t)(n * T_ * sizeof(T)), cudaMemcpyDeviceToDevice, s));
        if ((rc = axpby(A, V, -1.0, 1.0, T_, n, T_, s))) return rc;
        factor *= (double)(k + 1);
        if ((rc = axpby(S, A, ((k % 2) ? -1.0 : 1.0) / factor, 1.0, T_, n, T_, s))) return rc;
    }
    // D = E * S (into U)
    if ((rc = mul_rows(dtype, g, n, U, E, S, s))) return rc;

    // per-list recurrence: out[q] <- out[q] * E[item] + D[item], in list order
    RPYB_CUDA(cudaMemset2DAsync(out, (size_t)(ld_out * sizeof(T)), 0, (size_t)(T_ * sizeof(T)),
                                (size_t)n_lists, s));
    int64_t maxc = 0;
    for (int64_t q = 0; q < n_lists; ++q) maxc = std::max(maxc, off[q + 1] - off[q]);
    std::vector<int64_t> packed, pos(maxc + 1, 0);
    for (int64_t r = 0; r < maxc; ++r) {
        pos[r] = (int64_t)packed.size() / 2;
        std::vector<int64_t> qs, items;
        for (int64_t q = 0; q < n_lists; ++q)
            if (off[q + 1] - off[q] > r) {
                qs.push_back(q);
                items.push_back(off[q] + r);
            }
        packed.insert(packed.end(), qs.begin(), qs.end());
        packed.insert(packed.end(), items.begin(), items.end());
    }
    pos[maxc] = (int64_t)packed.size() / 2;
    if (packed.empty()) return RPYB_OK;
    int64_t* d_pk = reinterpret_cast<int64_t*>(rest);
    RPYB_CUDA(cudaMemcpyAsync(d_pk, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice, s));
    for (int64_t r = 0; r < maxc; ++r) {
        const int64_t m = pos[r + 1] - pos[r];
        const int64_t* q_idx = d_pk + 2 * pos[r];
        const int64_t* i_idx = q_idx + m;
        // V[i] <- out[q_i] * E[item_i]  (V has n >= m rows)
        ProductSpec sp;
        sp.klo = 1;
        sp.khi = g.depth;
        for (int k = 1; k <= g.depth; ++k) {
            sp.pmax[k] = k;
            sp.pmin[k] = 0;
            sp.scale[k] = 1.0;
        }
        sp.l0_write = true;
        sp.l0_prod = true;
        ProductRows rows;
        rows.out = V;
        rows.lhs = out;
        rows.rhs = E;
        rows.ld_out = T_;
        rows.ld_lhs = ld_out;
        rows.ld_rhs = T_;
        rows.lhs_idx = q_idx;
        rows.rhs_idx = i_idx;
        rows.batch = m;
        if ((rc = launch_product(dtype, g, sp, rows, s))) return rc;
        scatter_add_kernel<T><<<grid_of(m * T_), 256, 0, s>>>(out, ld_out, V, U, T_, q_idx, i_idx,
                                                               m);
        RPYB_CUDA(cudaGetLastError());
    }
    return RPYB_OK;
}

size_t bytes_for(int dtype, const Geometry& g, int64_t n_lists, int64_t n_items)
{
    const int64_t es = dtype == RPYB_F64 ? 8 : 4;
    const size_t rb = (size_t)((std::max<int64_t>(n_items, 1) * g.size() * es + 255) / 256 * 256);
    const int64_t ews = rpyb_ft_exp_workspace_size(dtype, g.width, g.depth, std::max<int64_t>(n_items, 1));
    (void)n_lists;
    return 6 * rb + (size_t)((std::max<int64_t>(ews, 1) + 255) / 256 * 256) +
           (size_t)((2 * n_items * 8 + 255) / 256 * 256);
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_sig_derivative_workspace_size(int dtype, int32_t width, int32_t depth,
                                                    int64_t n_lists, int64_t n_items)
{
    Geometry g;
    if ((dtype != RPYB_F32 && dtype != RPYB_F64) || make_geometry(width, depth, g) ||
        n_lists < 0 || n_items < 0)
        return -1;
    return (int64_t)bytes_for(dtype, g, n_lists, n_items);
}

RPYB_API int rpyb_sig_derivative(int dtype, int32_t width, int32_t depth, int64_t n_lists,
                                 const int64_t* offsets_host, const void* logsig,
                                 const void* perturbation, int64_t ld_lie, void* out,
                                 int64_t ld_out, void* workspace, size_t workspace_bytes,
                                 void* stream)
{
    int rc;
    if (dtype != RPYB_F32 && dtype != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported dtype");
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
    const int64_t lie_dim = rpyb_lie_basis_size(width, depth);
    if (lie_dim < 0) return (int)lie_dim;
    if (ld_out < g.size()) return fail(RPYB_E_INVALID, "ld_out too small");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n_items == 0) {
        const size_t es = dtype == RPYB_F64 ? 8 : 4;
        RPYB_CUDA(cudaMemset2DAsync(out, (size_t)ld_out * es, 0, (size_t)g.size() * es,
                                    (size_t)n_lists, s));
        return RPYB_OK;
    }
    if (!logsig || !perturbation) return fail(RPYB_E_INVALID, "null Lie arrays");
    if (ld_lie < lie_dim) return fail(RPYB_E_INVALID, "ld_lie smaller than the Lie dimension");

    const LieMapsDev* maps = nullptr;
    if ((rc = lie_maps_device(g, &maps))) return rc;
    const int64_t* d_ptr[2] = {maps->l2t_ptr, nullptr};
    const int64_t* d_idx[2] = {maps->l2t_idx, nullptr};
    const double* d_val[2] = {maps->l2t_val, nullptr};

    Scratch sc(workspace, workspace_bytes, s);
    void* ws = nullptr;
    if ((rc = sc.get(bytes_for(dtype, g, n_lists, n_items), &ws))) return rc;
    if (dtype == RPYB_F64)
        return derivative<double>(g, n_lists, offsets_host, static_cast<const double*>(logsig),
                                  static_cast<const double*>(perturbation), ld_lie,
                                  static_cast<double*>(out), ld_out, static_cast<char*>(ws), d_ptr,
                                  d_idx, d_val, lie_dim, s);
    return derivative<float>(g, n_lists, offsets_host, static_cast<const float*>(logsig),
                             static_cast<const float*>(perturbation), ld_lie,
                             static_cast<float*>(out), ld_out, static_cast<char*>(ws), d_ptr, d_idx,
                             d_val, lie_dim, s);
}

}  // extern "C"
