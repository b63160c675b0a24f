// Batched signatures straight from host memory: the increments are copied to
// the device, the signatures computed and copied back in chunks of streams,
// with the host->device copy of chunk i+1 and the device->host copy of chunk
// i-1 overlapping the kernel of chunk i (two copy streams, double-buffered
// device chunks).  Consecutive kernels alternate between two compute streams
// so that one chunk's kernel fills the tail of the previous one.  With pinned
// host buffers the PCIe transfers hide behind the computation.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "common.cuh"

namespace rpyb {
namespace {

struct CopyStreams {
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaStream_t comp = nullptr;   // second compute stream (odd chunks)
};

std::mutex g_cs_mu;
CopyStreams g_cs[64];

int copy_streams(CopyStreams** out)
{
    int dev = 0;
    RPYB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(RPYB_E_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lk(g_cs_mu);
    CopyStreams& c = g_cs[dev];
    if (!c.h2d) {
        RPYB_CUDA(cudaStreamCreateWithFlags(&c.h2d, cudaStreamNonBlocking));
        RPYB_CUDA(cudaStreamCreateWithFlags(&c.d2h, cudaStreamNonBlocking));
        RPYB_CUDA(cudaStreamCreateWithFlags(&c.comp, cudaStreamNonBlocking));
    }
    *out = &c;
    return RPYB_OK;
}

struct Chunk {
    int64_t s0, s1;       // streams [s0, s1)
    int64_t r0, r1;       // increment rows [r0, r1)
};

// Contiguous chunks of about equal total length, except that the first and
// the last carry half a share: the first kernel starts after a shorter
// upload and the last copy-out, which nothing overlaps, is shorter.
std::vector<Chunk> split(const int64_t* off, int64_t n, int chunks)
{
    std::vector<Chunk> out;
    const int64_t total = off[n];
    const double shares = chunks > 2 ? chunks - 1.0 : (double)chunks;
    int64_t s = 0;
    for (int c = 0; c < chunks && s < n; ++c) {
        const double done = chunks > 2 ? (c + 1 == chunks ? shares : c + 0.5) : c + 1.0;
        const int64_t target = (c + 1 == chunks) ? total : (int64_t)((double)total * done / shares);
        int64_t e = s + 1;
        while (e < n && off[e] < target) ++e;
        out.push_back({s, e, off[s], off[e]});
        s = e;
    }
    if (s < n) {
        out.back().s1 = n;
        out.back().r1 = off[n];
    }
    return out;
}

struct Layout {
    int64_t meta_bytes, inc_bytes, out_bytes, sig_ws_bytes, total;
};

Layout layout(int mode, int32_t width, const Geometry& g, const std::vector<Chunk>& ch,
              int64_t n_streams, int64_t sig_ws)
{
    const int64_t es = (mode == RPYB_F64) ? 8 : 4;
    int64_t max_rows = 0, max_streams = 0;
    for (const auto& c : ch) {
        max_rows = std::max(max_rows, c.r1 - c.r0);
        max_streams = std::max(max_streams, c.s1 - c.s0);
    }
    Layout l{};
    // per chunk: local offsets (s1-s0+1) and order (s1-s0)
    l.meta_bytes = ((2 * n_streams + (int64_t)ch.size()) * 8 + 255) / 256 * 256;
    l.inc_bytes = (max_rows * width * es + 255) / 256 * 256;
    l.out_bytes = (max_streams * g.size() * es + 255) / 256 * 256;
    l.sig_ws_bytes = (sig_ws + 255) / 256 * 256;
    l.total = l.meta_bytes + 2 * (l.inc_bytes + l.out_bytes + l.sig_ws_bytes);
    return l;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_signature_host_device_bytes(int mode, int32_t width, int32_t depth,
                                                  int64_t n_streams, const int64_t* offsets_host,
                                                  int32_t n_chunks)
{
    Geometry g;
    if (make_geometry(width, depth, g) || n_streams < 0 || !offsets_host || n_chunks < 1)
        return -1;
    const auto ch = split(offsets_host, n_streams, n_chunks);
    int64_t max_streams = 1;
    for (const auto& c : ch) max_streams = std::max(max_streams, c.s1 - c.s0);
    const int64_t ws = rpyb_signature_workspace_size(mode, width, depth, max_streams);
    if (ws < 0) return -1;
    return layout(mode, width, g, ch, n_streams, ws).total;
}

RPYB_API int rpyb_signature_host(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                 const int64_t* offsets_host, const void* inc_host,
                                 void* out_host, int64_t ld_out, int32_t n_chunks,
                                 void* device_buffer, size_t device_bytes, void* stream)
{
    int rc;
    if (mode != RPYB_F32 && mode != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported mode");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n_streams < 0 || n_chunks < 1) return fail(RPYB_E_INVALID, "invalid sizes");
    if (n_streams == 0) return RPYB_OK;
    if (!offsets_host || !inc_host || !out_host) return fail(RPYB_E_INVALID, "null pointer");
    if (offsets_host[0] != 0) return fail(RPYB_E_INVALID, "offsets must start at 0");
    for (int64_t s = 0; s < n_streams; ++s)
        if (offsets_host[s + 1] < offsets_host[s])
            return fail(RPYB_E_INVALID, "offsets must be non-decreasing");
    if (ld_out < g.size()) return fail(RPYB_E_INVALID, "ld_out too small");
    const int64_t need = rpyb_signature_host_device_bytes(mode, width, depth, n_streams,
                                                         offsets_host, n_chunks);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    Scratch scratch(device_buffer, device_bytes, cs);
    void* dev = nullptr;
    if ((rc = scratch.get((size_t)need, &dev))) return rc;

    const auto ch = split(offsets_host, n_streams, n_chunks);
    int64_t max_streams = 1;
    for (const auto& c : ch) max_streams = std::max(max_streams, c.s1 - c.s0);
    const int64_t sig_ws = rpyb_signature_workspace_size(mode, width, depth, max_streams);
    const Layout L = layout(mode, width, g, ch, n_streams, sig_ws);
    const int64_t es = (mode == RPYB_F64) ? 8 : 4;

    // chunk metadata: local offsets and longest-first order, uploaded once
    std::vector<int64_t> meta;
    std::vector<int64_t> meta_pos;
    for (const auto& c : ch) {
        meta_pos.push_back((int64_t)meta.size());
        for (int64_t s = c.s0; s <= c.s1; ++s) meta.push_back(offsets_host[s] - c.r0);
        std::vector<int64_t> ord(c.s1 - c.s0);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](int64_t x, int64_t y) {
            return (offsets_host[c.s0 + x + 1] - offsets_host[c.s0 + x]) >
                   (offsets_host[c.s0 + y + 1] - offsets_host[c.s0 + y]);
        });
        meta.insert(meta.end(), ord.begin(), ord.end());
    }
    char* base = static_cast<char*>(dev);
    int64_t* d_meta = reinterpret_cast<int64_t*>(base);
    RPYB_CUDA(cudaMemcpyAsync(d_meta, meta.data(), meta.size() * 8, cudaMemcpyHostToDevice, cs));
    // the host vector must outlive the copy
    RPYB_CUDA(cudaStreamSynchronize(cs));

    CopyStreams* cp = nullptr;
    if ((rc = copy_streams(&cp))) return rc;
    cudaEvent_t h2d_done[2], comp_done[2], d2h_done[2], start_ev;
    for (int i = 0; i < 2; ++i) {
        RPYB_CUDA(cudaEventCreateWithFlags(&h2d_done[i], cudaEventDisableTiming));
        RPYB_CUDA(cudaEventCreateWithFlags(&comp_done[i], cudaEventDisableTiming));
        RPYB_CUDA(cudaEventCreateWithFlags(&d2h_done[i], cudaEventDisableTiming));
    }
    RPYB_CUDA(cudaEventCreateWithFlags(&start_ev, cudaEventDisableTiming));
    // the copy streams start after everything already queued on the caller's stream
    RPYB_CUDA(cudaEventRecord(start_ev, cs));
    RPYB_CUDA(cudaStreamWaitEvent(cp->h2d, start_ev, 0));
    RPYB_CUDA(cudaStreamWaitEvent(cp->d2h, start_ev, 0));
    RPYB_CUDA(cudaStreamWaitEvent(cp->comp, start_ev, 0));

    int status = RPYB_OK;
    for (size_t i = 0; i < ch.size() && status == RPYB_OK; ++i) {
        const int b = (int)(i & 1);
        const Chunk& c = ch[i];
        char* inc_d = base + L.meta_bytes + b * (L.inc_bytes + L.out_bytes + L.sig_ws_bytes);
        char* out_d = inc_d + L.inc_bytes;
        char* ws_d = out_d + L.out_bytes;
        const int64_t ns = c.s1 - c.s0;
        // input buffer b is free once chunk i-2's kernel finished reading it
        if (i >= 2) RPYB_CUDA(cudaStreamWaitEvent(cp->h2d, comp_done[b], 0));
        RPYB_CUDA(cudaMemcpyAsync(inc_d,
                                  static_cast<const char*>(inc_host) + c.r0 * width * es,
                                  (size_t)((c.r1 - c.r0) * width * es), cudaMemcpyHostToDevice,
                                  cp->h2d));
        RPYB_CUDA(cudaEventRecord(h2d_done[b], cp->h2d));
        // consecutive chunks alternate between two compute streams, so a
        // chunk's kernel fills the tail of the previous one
        cudaStream_t ks = b ? cp->comp : cs;
        RPYB_CUDA(cudaStreamWaitEvent(ks, h2d_done[b], 0));
        // output buffer b is free once chunk i-2's copy-out finished
        if (i >= 2) RPYB_CUDA(cudaStreamWaitEvent(ks, d2h_done[b], 0));
        const int64_t* off_d = d_meta + meta_pos[i];
        const int64_t* ord_d = off_d + ns + 1;
        status = rpyb_signature(mode, width, depth, ns, off_d, inc_d, out_d, g.size(), ord_d,
                                ws_d, (size_t)L.sig_ws_bytes, ks);
        if (status != RPYB_OK) break;
        RPYB_CUDA(cudaEventRecord(comp_done[b], ks));
        RPYB_CUDA(cudaStreamWaitEvent(cp->d2h, comp_done[b], 0));
        RPYB_CUDA(cudaMemcpy2DAsync(static_cast<char*>(out_host) + c.s0 * ld_out * es,
                                    (size_t)(ld_out * es), out_d, (size_t)(g.size() * es),
                                    (size_t)(g.size() * es), (size_t)ns, cudaMemcpyDeviceToHost,
                                    cp->d2h));
        RPYB_CUDA(cudaEventRecord(d2h_done[b], cp->d2h));
    }
    // the caller's stream completes when the last copy-out has (which
    // follows every kernel)
    for (int i = 0; i < 2; ++i) RPYB_CUDA(cudaStreamWaitEvent(cs, d2h_done[i], 0));
    RPYB_CUDA(cudaEventRecord(start_ev, cp->comp));
    RPYB_CUDA(cudaStreamWaitEvent(cs, start_ev, 0));
    for (int i = 0; i < 2; ++i) {
        cudaEventDestroy(h2d_done[i]);
        cudaEventDestroy(comp_done[i]);
        cudaEventDestroy(d2h_done[i]);
    }
    cudaEventDestroy(start_ev);
    return status;
}

}  // extern "C"
