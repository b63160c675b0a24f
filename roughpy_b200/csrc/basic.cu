// Memory-bound companions of the product kernel: antipode, adjoint of left
// multiplication, and batched sparse (CSR) linear maps for Lie <-> tensor.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace rpyb {
namespace {

struct LevelTab {
    int64_t db[kMaxDepth + 2];
    int64_t pw[kMaxDepth + 1];
    int depth;
    int width;
};

__device__ __forceinline__ int level_of(const LevelTab& t, int64_t i)
{
    int k = 0;
    while (k < t.depth && i >= t.db[k + 1]) ++k;
    return k;
}

// out[rev(w)] = (-1)^k arg[w] per level; computed from the output side so
// that stores are coalesced (free_tensor_antipode.hpp:56-99).
template <typename T>
__global__ void antipode_kernel(T* out, const T* arg, int64_t ld_out, int64_t ld_arg,
                                int64_t batch, const LevelTab t)
{
    const int64_t size = t.db[t.depth + 1];
    const int64_t total = size * batch;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = g / size;
        const int64_t i = g - b * size;
        const int k = level_of(t, i);
        int64_t j = i - t.db[k];
        int64_t rev = 0;
        for (int q = 0; q < k; ++q) {
            rev = rev * t.width + (j % t.width);
            j /= t.width;
        }
        const T v = __ldg(arg + b * ld_arg + t.db[k] + rev);
        out[b * ld_out + i] = (k & 1) ? -v : v;
    }
}

// out_od[i] += sum_{q} sum_{j < d^q} op_q[j] * arg_{od+q}[j d^od + i]
// (free_tensor_adjoint_left_mul.hpp:43-75), one thread per output word,
// terms in the reference order (arg degree descending, op index ascending).
template <typename T>
__global__ void adjoint_left_mul_kernel(T* out, const T* op, const T* arg, int64_t ld_out,
                                        int64_t ld_op, int64_t ld_arg, int64_t batch,
                                        const LevelTab t, int out_max, int op_max, int arg_hi,
                                        int arg_lo)
{
    const int64_t size = t.db[out_max + 1];
    const int64_t total = size * batch;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = g / size;
        const int64_t iw = g - b * size;
        const int od = level_of(t, iw);
        const int64_t i = iw - t.db[od];
        const T* opr = op + b * ld_op;
        const T* ar = arg + b * ld_arg;
        T acc = out[b * ld_out + iw];
        double accd = 0.0;
        for (int ad = arg_hi; ad >= arg_lo; --ad) {
            const int q = ad - od;
            if (q < 0 || q > op_max) continue;
            const T* opq = opr + t.db[q];
            const T* arq = ar + t.db[ad] + i;
            const int64_t stride = t.pw[od];
            for (int64_t j = 0; j < t.pw[q]; ++j) {
                if constexpr (sizeof(T) == 8) acc = fma(__ldg(opq + j), __ldg(arq + j * stride), acc);
                else accd = fma((double)__ldg(opq + j), (double)__ldg(arq + j * stride), accd);
            }
        }
        if constexpr (sizeof(T) == 8) out[b * ld_out + iw] = acc;
        else out[b * ld_out + iw] = (T)((double)acc + accd);
    }
}

// y[b][r] += scale * sum_k val[k] * x[b][idx[k]]  (CSR), float64 accumulation;
// column indices outside [0, n_cols) are skipped.
template <typename T>
__global__ void csr_map_kernel(int64_t n_rows, int64_t n_cols, int64_t batch,
                               const int64_t* __restrict__ ptr,
                               const int64_t* __restrict__ idx, const double* __restrict__ val,
                               T* y, const T* x, int64_t ld_y, int64_t ld_x, double scale)
{
    const int64_t total = n_rows * batch;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = g / n_rows;
        const int64_t r = g - b * n_rows;
        const T* xr = x + b * ld_x;
        double acc = 0.0;
        for (int64_t k = __ldg(ptr + r), e = __ldg(ptr + r + 1); k < e; ++k) {
            const int64_t c = __ldg(idx + k);
            if ((uint64_t)c < (uint64_t)n_cols) acc = fma(__ldg(val + k), (double)__ldg(xr + c), acc);
        }
        T* yp = y + b * ld_y + r;
        *yp = (T)((double)*yp + scale * acc);
    }
}

LevelTab make_tab(const Geometry& g)
{
    LevelTab t{};
    for (int k = 0; k <= kMaxDepth + 1; ++k) t.db[k] = g.db[k];
    for (int k = 0; k <= kMaxDepth; ++k) t.pw[k] = g.pw[k];
    t.depth = g.depth;
    t.width = g.width;
    return t;
}

unsigned grid_for(int64_t total, int threads)
{
    const int64_t b = (total + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 64));
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int rpyb_ft_antipode(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                              const void* arg, int64_t ld_out, int64_t ld_arg, void* stream)
{
    int rc;
    if (dtype != RPYB_F32 && dtype != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported dtype");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !arg) return fail(RPYB_E_INVALID, "null tensor pointer");
    if (batch > 1 && (ld_out < g.size() || ld_arg < g.size()))
        return fail(RPYB_E_INVALID, "row stride smaller than the tensor size");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const LevelTab t = make_tab(g);
    const int threads = 256;
    const unsigned blocks = grid_for(g.size() * batch, threads);
    if (dtype == RPYB_F64)
        antipode_kernel<double><<<blocks, threads, 0, s>>>(
            static_cast<double*>(out), static_cast<const double*>(arg), ld_out, ld_arg, batch, t);
    else
        antipode_kernel<float><<<blocks, threads, 0, s>>>(
            static_cast<float*>(out), static_cast<const float*>(arg), ld_out, ld_arg, batch, t);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

RPYB_API int rpyb_ft_adjoint_left_mul(int dtype, int32_t width, int32_t depth, int64_t batch,
                                      void* out, const void* op, const void* arg, int64_t ld_out,
                                      int64_t ld_op, int64_t ld_arg, const int32_t* deg,
                                      void* stream)
{
    int rc;
    if (dtype != RPYB_F32 && dtype != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported dtype");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !op || !arg) return fail(RPYB_E_INVALID, "null tensor pointer");
    if (batch > 1 && (ld_out < g.size() || ld_op < g.size() || ld_arg < g.size()))
        return fail(RPYB_E_INVALID, "row stride smaller than the tensor size");
    int32_t b[3] = {-1, -1, -1};
    if (deg) std::memcpy(b, deg, sizeof(b));
    const int out_max = clamp_max_degree(b[0], depth);
    const int op_max = clamp_max_degree(b[1], depth);
    const int arg_max = clamp_max_degree(b[2], depth);
    // free_tensor_adjoint_left_mul.hpp:43-44 with all min degrees 0
    const int arg_hi = std::min(arg_max - 0, out_max);
    const int arg_lo = std::max(0 - op_max, 0);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const LevelTab t = make_tab(g);
    const int threads = 256;
    const unsigned blocks = grid_for(g.db[out_max + 1] * batch, threads);
    if (dtype == RPYB_F64)
        adjoint_left_mul_kernel<double><<<blocks, threads, 0, s>>>(
            static_cast<double*>(out), static_cast<const double*>(op),
            static_cast<const double*>(arg), ld_out, ld_op, ld_arg, batch, t, out_max, op_max,
            arg_hi, arg_lo);
    else
        adjoint_left_mul_kernel<float><<<blocks, threads, 0, s>>>(
            static_cast<float*>(out), static_cast<const float*>(op),
            static_cast<const float*>(arg), ld_out, ld_op, ld_arg, batch, t, out_max, op_max,
            arg_hi, arg_lo);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

RPYB_API int rpyb_sparse_map(int dtype, int64_t n_rows, int64_t n_cols, int64_t batch,
                             const int64_t* indptr, const int64_t* indices, const double* values,
                             void* y, const void* x, int64_t ld_y, int64_t ld_x, double scale,
                             void* stream)
{
    if (dtype != RPYB_F32 && dtype != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported dtype");
    if (n_rows < 0 || n_cols < 0 || batch < 0) return fail(RPYB_E_INVALID, "negative size");
    if (batch == 0 || n_rows == 0) return RPYB_OK;
    if (!indptr || !y || !x) return fail(RPYB_E_INVALID, "null pointer");
    if (batch > 1 && (ld_y < n_rows || ld_x < n_cols))
        return fail(RPYB_E_INVALID, "row stride smaller than the vector size");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int threads = 256;
    const unsigned blocks = grid_for(n_rows * batch, threads);
    if (dtype == RPYB_F64)
        csr_map_kernel<double><<<blocks, threads, 0, s>>>(n_rows, n_cols, batch, indptr, indices, values,
                                                         static_cast<double*>(y),
                                                         static_cast<const double*>(x), ld_y,
                                                         ld_x, scale);
    else
        csr_map_kernel<float><<<blocks, threads, 0, s>>>(n_rows, n_cols, batch, indptr, indices, values,
                                                        static_cast<float*>(y),
                                                        static_cast<const float*>(x), ld_y, ld_x,
                                                        scale);
    RPYB_CUDA(cudaGetLastError());
    return RPYB_OK;
}

}  // extern "C"
