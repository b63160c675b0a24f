// Host side of the dense free-tensor operations: argument checking, degree
// bounds (with roughpy.compute's semantics) and the Horner drivers for exp,
// fmexp and log, all expressed as launches of the batched product kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"
#include "product.cuh"

namespace rpyb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg)
{
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t err, const char* what)
{
    set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return (err == cudaErrorMemoryAllocation) ? RPYB_E_NOMEM : RPYB_E_CUDA;
}

int make_geometry(int32_t width, int32_t depth, Geometry& g)
{
    if (width < 1) return fail(RPYB_E_INVALID, "width must be >= 1");
    if (depth < 0 || depth > kMaxDepth)
        return fail(RPYB_E_INVALID, "depth must be in [0, " + std::to_string(kMaxDepth) + "]");
    g = Geometry{};
    g.width = width;
    g.depth = depth;
    g.pw[0] = 1;
    g.db[0] = 0;
    for (int k = 0; k <= depth; ++k) {
        if (k > 0) {
            if (g.pw[k - 1] > (int64_t(1) << 40) / width)
                return fail(RPYB_E_INVALID, "tensor too large");
            g.pw[k] = g.pw[k - 1] * width;
        }
        g.db[k + 1] = g.db[k] + g.pw[k];
    }
    if (g.db[depth + 1] >= (int64_t(1) << 31))
        return fail(RPYB_E_INVALID, "tensor has more than 2^31 scalars");
    for (int k = depth + 1; k <= kMaxDepth; ++k) g.pw[k] = g.pw[depth];
    for (int k = depth + 2; k <= kMaxDepth + 1; ++k) g.db[k] = g.db[depth + 1];
    return RPYB_OK;
}

// Library-owned stream-ordered memory pool per device.  Freed scratch stays
// in the pool (release threshold: unlimited) so that repeated calls with
// gigabyte temporaries do not map and unmap device memory each time;
// rpyb_release_cached_memory returns it to the driver.
namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
}  // namespace

static int scratch_pool(cudaMemPool_t* out)
{
    int dev = 0;
    RPYB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(RPYB_E_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        RPYB_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t threshold = UINT64_MAX;
        RPYB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return RPYB_OK;
}

Scratch::~Scratch()
{
    if (owned_) cudaFreeAsync(owned_, s_);
}

int Scratch::get(size_t bytes, void** p)
{
    if (bytes == 0) {
        *p = nullptr;
        return RPYB_OK;
    }
    if (ws_) {
        if (cap_ < bytes)
            return fail(RPYB_E_NOMEM, "workspace too small: need " + std::to_string(bytes) +
                                          " bytes, got " + std::to_string(cap_));
        *p = ws_;
        return RPYB_OK;
    }
    cudaMemPool_t pool = nullptr;
    int rc;
    if ((rc = scratch_pool(&pool))) return rc;
    RPYB_CUDA(cudaMallocFromPoolAsync(&owned_, bytes, pool, s_));
    *p = owned_;
    return RPYB_OK;
}

static size_t elem_size(int dtype) { return dtype == RPYB_F64 ? 8 : 4; }

static int check_dtype(int dtype)
{
    if (dtype != RPYB_F32 && dtype != RPYB_F64)
        return fail(RPYB_E_INVALID, "unsupported dtype (expected RPYB_F32 or RPYB_F64)");
    return RPYB_OK;
}

static int check_ld(int64_t ld, int64_t need, const char* name, int64_t batch)
{
    if (batch > 1 && ld < need)
        return fail(RPYB_E_INVALID, std::string(name) + " row stride smaller than the tensor size");
    return RPYB_OK;
}

// Degree-bound clamp matching roughpy/compute/_src/call_config.cpp:11-31.
static int clamp_bounds(int32_t& mn, int32_t& mx, int32_t depth, int arg)
{
    mx = clamp_max_degree(mx, depth);
    if (mn < 0) mn = 0;
    if (mn > mx)
        return fail(RPYB_E_INVALID, "invalid degree bounds for argument " + std::to_string(arg) +
                                        ": min_degree must not exceed max_degree");
    return RPYB_OK;
}

static int horner_buffers(int dtype, const Geometry& g, int64_t batch, int nbuf,
                          int64_t* bytes)
{
    *bytes = (int64_t)nbuf * batch * g.size() * (int64_t)elem_size(dtype);
    return RPYB_OK;
}

}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int rpyb_release_cached_memory(void)
{
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (int d = 0; d < 64; ++d)
        if (g_pools[d]) RPYB_CUDA(cudaMemPoolTrimTo(g_pools[d], 0));
    return RPYB_OK;
}

RPYB_API int rpyb_scratch_pool_usage(int64_t* used_bytes, int64_t* reserved_bytes)
{
    int dev = 0;
    RPYB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(RPYB_E_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lk(g_pool_mu);
    uint64_t used = 0, reserved = 0;
    if (g_pools[dev]) {
        RPYB_CUDA(cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrUsedMemCurrent, &used));
        RPYB_CUDA(cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrReservedMemCurrent,
                                          &reserved));
    }
    if (used_bytes) *used_bytes = (int64_t)used;
    if (reserved_bytes) *reserved_bytes = (int64_t)reserved;
    return RPYB_OK;
}

RPYB_API const char* rpyb_last_error(void) { return rpyb::g_last_error.c_str(); }

RPYB_API const char* rpyb_version(void) { return "roughpy_b200 0.1.0 (sm_100a)"; }

RPYB_API int64_t rpyb_tensor_size(int32_t width, int32_t depth)
{
    Geometry g;
    if (make_geometry(width, depth, g) != RPYB_OK) return -1;
    return g.size();
}

RPYB_API int rpyb_ft_fma(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                         const void* lhs, const void* rhs, int64_t ld_out, int64_t ld_lhs,
                         int64_t ld_rhs, const int32_t* deg_bounds, void* stream)
{
    int rc;
    if ((rc = check_dtype(dtype))) return rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !lhs || !rhs) return fail(RPYB_E_INVALID, "null tensor pointer");
    if ((rc = check_ld(ld_out, g.size(), "out", batch))) return rc;
    if ((rc = check_ld(ld_lhs, g.size(), "lhs", batch))) return rc;
    if ((rc = check_ld(ld_rhs, g.size(), "rhs", batch))) return rc;
    int32_t b[6] = {0, -1, 0, -1, 0, -1};
    if (deg_bounds) std::memcpy(b, deg_bounds, sizeof(b));
    for (int i = 0; i < 3; ++i)
        if ((rc = clamp_bounds(b[2 * i], b[2 * i + 1], depth, i))) return rc;
    const int out_min = b[0], out_max = b[1], lmin = b[2], lmax = b[3], rmin = b[4], rmax = b[5];

    // free_tensor_fma.hpp:24-51
    ProductSpec sp;
    sp.klo = std::max(1, out_min);
    sp.khi = out_max;
    for (int k = sp.klo; k <= sp.khi; ++k) {
        sp.pmax[k] = std::min(lmax, k - rmin);
        sp.pmin[k] = std::max(lmin, k - rmax);
        sp.scale[k] = 1.0;
    }
    sp.accumulate = true;
    if (out_min == 0 && lmin == 0 && rmin == 0) {
        sp.l0_write = true;
        sp.l0_base = 1;
        sp.l0_prod = true;
        sp.scale0 = 1.0;
    }
    ProductRows rows;
    rows.out = out;
    rows.lhs = lhs;
    rows.rhs = rhs;
    rows.ld_out = ld_out;
    rows.ld_lhs = ld_lhs;
    rows.ld_rhs = ld_rhs;
    rows.batch = batch;
    return launch_product(dtype, g, sp, rows, static_cast<cudaStream_t>(stream));
}

RPYB_API int rpyb_ft_mul_gather(int dtype, int32_t width, int32_t depth, int64_t n, void* out,
                                const void* lhs, const void* rhs, int64_t ld,
                                const int64_t* out_idx, const int64_t* lhs_idx,
                                const int64_t* rhs_idx, int accumulate, void* stream)
{
    int rc;
    if ((rc = check_dtype(dtype))) return rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (n == 0) return RPYB_OK;
    if (!out || !lhs || !rhs) return fail(RPYB_E_INVALID, "null tensor pointer");
    if (ld < g.size()) return fail(RPYB_E_INVALID, "row stride smaller than the tensor size");
    ProductSpec sp;
    sp.klo = 1;
    sp.khi = depth;
    for (int k = 1; k <= depth; ++k) {
        sp.pmax[k] = k;
        sp.pmin[k] = 0;
        sp.scale[k] = 1.0;
    }
    sp.accumulate = accumulate != 0;
    sp.l0_write = true;
    sp.l0_base = accumulate ? 1 : 0;
    sp.l0_prod = true;
    ProductRows rows;
    rows.out = out;
    rows.lhs = lhs;
    rows.rhs = rhs;
    rows.ld_out = rows.ld_lhs = rows.ld_rhs = ld;
    rows.out_idx = out_idx;
    rows.lhs_idx = lhs_idx;
    rows.rhs_idx = rhs_idx;
    rows.batch = n;
    return launch_product(dtype, g, sp, rows, static_cast<cudaStream_t>(stream));
}

RPYB_API int rpyb_ft_mul_gather_mixed(int32_t width, int32_t depth, int64_t n, double* out,
                                      const double* lhs, const float* rhs, int64_t ld,
                                      const int64_t* out_idx, const int64_t* lhs_idx,
                                      const int64_t* rhs_idx, int accumulate, void* stream)
{
    int rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (n == 0) return RPYB_OK;
    if (!out || !lhs || !rhs) return fail(RPYB_E_INVALID, "null tensor pointer");
    if (ld < g.size()) return fail(RPYB_E_INVALID, "row stride smaller than the tensor size");
    ProductSpec sp;
    sp.klo = 1;
    sp.khi = depth;
    for (int k = 1; k <= depth; ++k) {
        sp.pmax[k] = k;
        sp.pmin[k] = 0;
        sp.scale[k] = 1.0;
    }
    sp.accumulate = accumulate != 0;
    sp.l0_write = true;
    sp.l0_base = accumulate ? 1 : 0;
    sp.l0_prod = true;
    ProductRows rows;
    rows.out = out;
    rows.lhs = lhs;
    rows.rhs = rhs;
    rows.ld_out = rows.ld_lhs = rows.ld_rhs = ld;
    rows.out_idx = out_idx;
    rows.lhs_idx = lhs_idx;
    rows.rhs_idx = rhs_idx;
    rows.batch = n;
    return launch_product(kMixedF64F32, g, sp, rows, static_cast<cudaStream_t>(stream));
}

RPYB_API int64_t rpyb_ft_inplace_mul_workspace_size(int dtype, int32_t width, int32_t depth,
                                                    int64_t batch)
{
    Geometry g;
    if (check_dtype(dtype) || make_geometry(width, depth, g)) return -1;
    int64_t bytes;
    horner_buffers(dtype, g, batch, 1, &bytes);
    return bytes;
}

RPYB_API int rpyb_ft_inplace_mul(int dtype, int32_t width, int32_t depth, int64_t batch,
                                 void* lhs, const void* rhs, int64_t ld_lhs, int64_t ld_rhs,
                                 const int32_t* deg_bounds, void* workspace,
                                 size_t workspace_bytes, void* stream)
{
    int rc;
    if ((rc = check_dtype(dtype))) return rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!lhs || !rhs) return fail(RPYB_E_INVALID, "null tensor pointer");
    if ((rc = check_ld(ld_lhs, g.size(), "lhs", batch))) return rc;
    if ((rc = check_ld(ld_rhs, g.size(), "rhs", batch))) return rc;
    int32_t b[4] = {0, -1, 0, -1};
    if (deg_bounds) std::memcpy(b, deg_bounds, sizeof(b));
    for (int i = 0; i < 2; ++i)
        if ((rc = clamp_bounds(b[2 * i], b[2 * i + 1], depth, i))) return rc;
    const int lmin = b[0], lmax = b[1], rmin = b[2], rmax = b[3];
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    const int64_t T = g.size();
    const size_t es = elem_size(dtype);
    Scratch scratch(workspace, workspace_bytes, s);
    void* tmp = nullptr;
    if ((rc = scratch.get((size_t)(batch * T) * es, &tmp))) return rc;

    // free_tensor_inplace_mul.hpp:22-85, written out of place into tmp.
    ProductSpec sp;
    sp.klo = std::max(1, lmin);
    sp.khi = lmax;
    for (int k = sp.klo; k <= sp.khi; ++k) {
        sp.pmax[k] = k - rmin;
        sp.pmin[k] = std::max(lmin, k - rmax);
        sp.scale[k] = 1.0;
    }
    if (lmin == 0) {
        sp.l0_write = true;
        sp.l0_base = 0;
        sp.l0_prod = (rmin == 0);
    }
    ProductRows rows;
    rows.out = tmp;
    rows.ld_out = T;
    rows.lhs = lhs;
    rows.ld_lhs = ld_lhs;
    rows.rhs = rhs;
    rows.ld_rhs = ld_rhs;
    rows.batch = batch;
    if ((rc = launch_product(dtype, g, sp, rows, s))) return rc;
    const int64_t c0 = g.db[lmin], c1 = g.db[lmax + 1];
    RPYB_CUDA(cudaMemcpy2DAsync(static_cast<char*>(lhs) + c0 * es, (size_t)ld_lhs * es,
                                static_cast<char*>(tmp) + c0 * es, (size_t)T * es,
                                (size_t)(c1 - c0) * es, (size_t)batch, cudaMemcpyDeviceToDevice,
                                s));
    return RPYB_OK;
}

RPYB_API int64_t rpyb_ft_exp_workspace_size(int dtype, int32_t width, int32_t depth,
                                            int64_t batch)
{
    return rpyb_ft_inplace_mul_workspace_size(dtype, width, depth, batch);
}

RPYB_API int64_t rpyb_ft_fmexp_workspace_size(int dtype, int32_t width, int32_t depth,
                                              int64_t batch)
{
    return rpyb_ft_inplace_mul_workspace_size(dtype, width, depth, batch);
}

RPYB_API int64_t rpyb_ft_log_workspace_size(int dtype, int32_t width, int32_t depth,
                                            int64_t batch)
{
    Geometry g;
    if (check_dtype(dtype) || make_geometry(width, depth, g)) return -1;
    int64_t bytes;
    horner_buffers(RPYB_F64, g, batch, dtype == RPYB_F64 ? 1 : 3, &bytes);
    return bytes;
}

// Horner series driver shared by exp and fmexp: steps deg = M..1 with
// max_level = M - deg + 1 (free_tensor_exp.hpp:26-35, free_tensor_fmexp.hpp:31-38).
// The last step writes `out`; earlier steps alternate with `tmp`.
static int horner_exp_like(int dtype, const Geometry& g, int M, int64_t batch, void* out,
                           int64_t ld_out, const void* first_cur, int64_t ld_first,
                           const void* arg, int64_t ld_arg, const void* addend,
                           int64_t ld_add, void* tmp, cudaStream_t s)
{
    const int64_t T = g.size();
    for (int step = 1; step <= M; ++step) {
        const int deg = M - step + 1;
        const int ml = M - deg + 1;
        const bool dst_is_out = ((M - step) % 2) == 0;
        void* dst = dst_is_out ? out : tmp;
        const int64_t ld_dst = dst_is_out ? ld_out : T;
        const void* cur;
        int64_t ld_cur;
        if (step == 1) {
            cur = first_cur;
            ld_cur = ld_first;
        } else {
            cur = dst_is_out ? tmp : out;
            ld_cur = dst_is_out ? T : ld_out;
        }
        ProductSpec sp;
        sp.klo = 1;
        sp.khi = ml;
        for (int k = 1; k <= ml; ++k) {
            sp.pmax[k] = k - 1;
            sp.pmin[k] = 0;
            sp.scale[k] = 1.0 / (double)deg;
        }
        sp.l0_write = true;
        if (addend) {
            // fmexp: level 0 becomes multiplier[0]; L0 read from the current rows
            sp.l0_base = 2;
            sp.lhs0_from_mem = true;
        } else {
            // exp: level 0 is reset to the unit; L0 == 1
            sp.l0_base = 0;
            sp.l0_const = 1.0;
            sp.lhs0_from_mem = false;
            sp.lhs0_add = 1.0;
        }
        ProductRows rows;
        rows.out = dst;
        rows.ld_out = ld_dst;
        rows.lhs = cur;
        rows.ld_lhs = ld_cur;
        rows.rhs = arg;
        rows.ld_rhs = ld_arg;
        rows.addend = addend;
        rows.ld_add = ld_add;
        rows.batch = batch;
        int rc = launch_product(dtype, g, sp, rows, s);
        if (rc) return rc;
    }
    return RPYB_OK;
}

RPYB_API int rpyb_ft_exp(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                         const void* arg, int64_t ld_out, int64_t ld_arg, int32_t out_depth,
                         void* workspace, size_t workspace_bytes, void* stream)
{
    int rc;
    if ((rc = check_dtype(dtype))) return rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !arg) return fail(RPYB_E_INVALID, "null tensor pointer");
    if ((rc = check_ld(ld_out, g.size(), "out", batch))) return rc;
    if ((rc = check_ld(ld_arg, g.size(), "arg", batch))) return rc;
    const int M = clamp_max_degree(out_depth, depth);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (M == 0) {
        // only the unit: out[0] = 1
        ProductSpec sp;
        sp.khi = 0;
        sp.l0_write = true;
        sp.l0_const = 1.0;
        ProductRows rows;
        rows.out = out;
        rows.ld_out = ld_out;
        rows.lhs = arg;
        rows.ld_lhs = ld_arg;
        rows.rhs = arg;
        rows.ld_rhs = ld_arg;
        rows.batch = batch;
        return launch_product(dtype, g, sp, rows, s);
    }
    Scratch scratch(workspace, workspace_bytes, s);
    void* tmp = nullptr;
    if (M > 1 &&
        (rc = scratch.get((size_t)(batch * g.size()) * elem_size(dtype), &tmp)))
        return rc;
    return horner_exp_like(dtype, g, M, batch, out, ld_out, out, ld_out, arg, ld_arg, nullptr,
                           0, tmp, s);
}

RPYB_API int rpyb_ft_fmexp(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                           const void* multiplier, const void* exponent, int64_t ld_out,
                           int64_t ld_mul, int64_t ld_exp, int32_t out_depth, void* workspace,
                           size_t workspace_bytes, void* stream)
{
    int rc;
    if ((rc = check_dtype(dtype))) return rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !multiplier || !exponent) return fail(RPYB_E_INVALID, "null tensor pointer");
    if ((rc = check_ld(ld_out, g.size(), "out", batch))) return rc;
    if ((rc = check_ld(ld_mul, g.size(), "multiplier", batch))) return rc;
    if ((rc = check_ld(ld_exp, g.size(), "exponent", batch))) return rc;
    const int M = clamp_max_degree(out_depth, depth);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t es = elem_size(dtype);
    if (M == 0) {
        RPYB_CUDA(cudaMemcpy2DAsync(out, (size_t)ld_out * es, multiplier, (size_t)ld_mul * es, es,
                                    (size_t)batch, cudaMemcpyDeviceToDevice, s));
        return RPYB_OK;
    }
    Scratch scratch(workspace, workspace_bytes, s);
    void* tmp = nullptr;
    if (M > 1 && (rc = scratch.get((size_t)(batch * g.size()) * es, &tmp))) return rc;
    return horner_exp_like(dtype, g, M, batch, out, ld_out, multiplier, ld_mul, exponent, ld_exp,
                           multiplier, ld_mul, tmp, s);
}

RPYB_API int rpyb_ft_log(int dtype, int32_t width, int32_t depth, int64_t batch, void* out,
                         const void* arg, int64_t ld_out, int64_t ld_arg, int32_t out_depth,
                         int32_t arg_depth, void* workspace, size_t workspace_bytes, void* stream)
{
    int rc;
    if ((rc = check_dtype(dtype))) return rc;
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (batch < 0) return fail(RPYB_E_INVALID, "negative batch");
    if (batch == 0) return RPYB_OK;
    if (!out || !arg) return fail(RPYB_E_INVALID, "null tensor pointer");
    if ((rc = check_ld(ld_out, g.size(), "out", batch))) return rc;
    if ((rc = check_ld(ld_arg, g.size(), "arg", batch))) return rc;
    const int M = clamp_max_degree(out_depth, depth);
    const int Ma = clamp_max_degree(arg_depth, depth);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t T = g.size();

    Scratch scratch(workspace, workspace_bytes, s);
    void* base = nullptr;
    const int nbuf = (dtype == RPYB_F64) ? 1 : 3;
    if ((rc = scratch.get((size_t)(nbuf * batch * T) * 8, &base))) return rc;
    double* tmp = static_cast<double*>(base);
    double* out64 = static_cast<double*>(out);
    const double* arg64 = static_cast<const double*>(arg);
    int64_t ld_o = ld_out, ld_a = ld_arg;
    if (dtype == RPYB_F32) {
        double* a64 = tmp + batch * T;
        double* o64 = tmp + 2 * batch * T;
        if ((rc = launch_convert_rows(RPYB_F64, a64, T, RPYB_F32, arg, ld_arg, T, batch, s)))
            return rc;
        if ((rc = launch_convert_rows(RPYB_F64, o64, T, RPYB_F32, out, ld_out, T, batch, s)))
            return rc;
        arg64 = a64;
        out64 = o64;
        ld_o = ld_a = T;
    }

    // free_tensor_log.hpp:23-38.  The coefficient added to out[0] before each
    // multiply enters as the level-0 value of the current rows.  When the
    // first step writes `out` itself, the incoming out[0] is first parked in
    // the other buffer so that no launch reads the rows it writes.
    if (M >= 1 && ((M - 1) % 2) == 0) {
        RPYB_CUDA(cudaMemcpy2DAsync(tmp, (size_t)T * 8, out64, (size_t)ld_o * 8, 8,
                                    (size_t)batch, cudaMemcpyDeviceToDevice, s));
    }
    for (int step = 1; step <= M; ++step) {
        const int deg = M - step + 1;
        const int ml = M - deg + 1;
        const double coeff = (deg % 2 == 0) ? -(1.0 / (double)deg) : (1.0 / (double)deg);
        const bool dst_is_out = ((M - step) % 2) == 0;
        double* dst = dst_is_out ? out64 : tmp;
        const int64_t ld_dst = dst_is_out ? ld_o : T;
        const double* cur = dst_is_out ? tmp : out64;
        const int64_t ld_cur = dst_is_out ? T : ld_o;
        const int rmax = std::min(Ma, ml);
        ProductSpec sp;
        sp.klo = 1;
        sp.khi = ml;
        for (int k = 1; k <= ml; ++k) {
            sp.pmax[k] = k - 1;
            sp.pmin[k] = std::max(0, k - rmax);
            sp.scale[k] = 1.0;
        }
        sp.lhs0_from_mem = (step == 1);
        sp.lhs0_add = coeff;
        sp.l0_write = true;
        sp.l0_base = 0;
        ProductRows rows;
        rows.out = dst;
        rows.ld_out = ld_dst;
        rows.lhs = cur;
        rows.ld_lhs = ld_cur;
        rows.rhs = arg64;
        rows.ld_rhs = ld_a;
        rows.batch = batch;
        if ((rc = launch_product(RPYB_F64, g, sp, rows, s))) return rc;
    }
    // M == 0: the series is empty and out keeps its contents.
    if (dtype == RPYB_F32) {
        if ((rc = launch_convert_rows(RPYB_F32, out, ld_out, RPYB_F64, out64, T, T, batch, s)))
            return rc;
    }
    return RPYB_OK;
}

}  // extern "C"
