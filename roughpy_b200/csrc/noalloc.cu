// rpyb_ft_exp_noalloc: the tensor exponential for callers that must not
// allocate device memory.
//
// Some callers cannot call cudaMalloc.  Examples are code that runs under a
// host application which owns every device allocation (a fixed, pre-sized
// memory pool or budget), code on a latency-critical thread where an
// allocation or free would synchronise the device, and plugins called back
// from another library that forbids allocation inside the callback.  For
// them this entry point takes its Horner ping-pong buffer from a file-scope
// device array instead of a workspace argument.
//
// The array below is a fixed kNoAllocScratchBytes (8 MiB) on every GPU that
// loads this library, held until the process exits.  Calls whose scratch
// need exceeds it are rejected with RPYB_E_INVALID before anything runs.
//
// In host code `g_exp_scratch` names a host-side shadow, not device memory,
// so its device address is fetched with cudaGetSymbolAddress, once per device
// with that device current, on the first call made on that device.  Make
// that first call before any stream capture begins.
//
// Every call on a device shares the same array and it keeps the previous
// call's contents.  The exp Horner series writes each part of the buffer
// before reading it within one call, so nothing needs clearing.  Calls that
// overlap on the GPU (for example on two streams without ordering between
// them) race on the array: order them on one stream or with events.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"

namespace rpyb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_exp_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

int scratch_for_current_device(void** out)
{
    int dev = 0;
    RPYB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(RPYB_E_UNSUPPORTED, "device ordinal beyond the static scratch table");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_exp_scratch);
        if (err != cudaSuccess) return cuda_fail(err, "cudaGetSymbolAddress(g_exp_scratch)");
        if (p == nullptr) return fail(RPYB_E_CUDA, "static scratch has no device address");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return RPYB_OK;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_ft_exp_noalloc_max_bytes(void) { return (int64_t)kNoAllocScratchBytes; }

RPYB_API int rpyb_ft_exp_noalloc(int dtype, int32_t width, int32_t depth, int64_t batch,
                                 void* out, const void* arg, int64_t ld_out, int64_t ld_arg,
                                 int32_t out_depth, void* stream)
{
    if (batch < 0) return fail(RPYB_E_INVALID, "rpyb_ft_exp_noalloc: negative batch");
    // bound the batch by division first: the byte count of a huge batch
    // would overflow int64 and could pass a product-based check
    const int64_t per_row = rpyb_ft_exp_workspace_size(dtype, width, depth, 1);
    if (per_row <= 0) return fail(RPYB_E_INVALID, "invalid dtype, width or depth");
    if (batch > (int64_t)kNoAllocScratchBytes / per_row)
        return fail(RPYB_E_INVALID,
                    "rpyb_ft_exp_noalloc: batch " + std::to_string(batch) + " needs more than the " +
                        "8 MiB static scratch (" + std::to_string(per_row) + " bytes per row)");
    const int64_t need = rpyb_ft_exp_workspace_size(dtype, width, depth, batch);
    if (need < 0 || (size_t)need > kNoAllocScratchBytes)
        return fail(RPYB_E_INVALID, "rpyb_ft_exp_noalloc: scratch size out of range");
    if (batch <= 0) return rpyb_ft_exp(dtype, width, depth, batch, out, arg, ld_out, ld_arg,
                                       out_depth, nullptr, 0, stream);
    void* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    return rpyb_ft_exp(dtype, width, depth, batch, out, arg, ld_out, ld_arg, out_depth, scratch,
                       kNoAllocScratchBytes, stream);
}

}  // extern "C"
