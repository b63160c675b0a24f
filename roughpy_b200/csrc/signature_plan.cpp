// Signature plans: one batch layout (stream lengths known on the host),
// its launch schedule and the device memory it needs, reused across calls.
//
// A schedule has three knobs:
//   * g    -- lane shape of the kernel (level-(N-1) words per lane);
//   * wpb  -- warps per block (0: the occupancy-best block size);
//   * seg  -- time-segment length for long streams (0: never split).
// Splitting uses the associativity of the Chen product: a stream longer than
// `seg` is cut into k balanced segments, every segment becomes its own work
// item of the persistent kernel (so a handful of very long streams still
// fills the GPU), and the k segment signatures are multiplied back together
// in order by a pairwise tree of batched free-tensor products.  The
// reference computes a stream's signature as one left-to-right chain of
// fmexp steps (algebra/src/lite_context.h:542-563); the tree evaluates the
// same product in another association.
//
// The schedule is chosen per key (device, mode, width, depth, log2 of the
// longest stream, log2 of the batch size): from RPYB_SIG_SCHEDULE when set,
// else from the JSON cache (RPYB_SIG_TUNE_CACHE, default
// $XDG_CACHE_HOME/roughpy_b200/signature_schedules.json), else -- when the
// caller allows it -- by timing the candidates on synthetic increments of
// the plan's own layout, and the winner is written back to the cache.
#include <fcntl.h>
#include <sys/file.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "signature_internal.cuh"

namespace rpyb {
namespace {

struct Schedule {
    int g = 0;
    int wpb = 0;
    int64_t seg = 0;
    double ms = -1.0;     // measured time of the tuning run (-1: not measured)
    std::string source = "default";
};

struct DeviceBuf {
    void* p = nullptr;
    ~DeviceBuf() { if (p) cudaFree(p); }
    int alloc(size_t bytes)
    {
        if (p) { cudaFree(p); p = nullptr; }
        if (bytes == 0) return RPYB_OK;
        RPYB_CUDA(cudaMalloc(&p, bytes));
        return RPYB_OK;
    }
};

// Pseudo-random increments for timing runs: uniform in +-sqrt(3/len_mean),
// the variance of the N(0, 1/len) increments of a unit-variance path.
__global__ void synthetic_rows_kernel(void* out, int64_t n, int f64, double scale)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
        h ^= h >> 31;
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 29;
        const double u = ((double)(h >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
        if (f64) static_cast<double*>(out)[i] = u * scale;
        else static_cast<float*>(out)[i] = (float)(u * scale);
    }
}

// out row dst[i] <- scratch row src[i] (the merged signatures of split streams)
__global__ void copy_rows_kernel(const char* __restrict__ src, int64_t ld_src, char* __restrict__ dst,
                                 int64_t ld_dst, const int64_t* __restrict__ src_idx,
                                 const int64_t* __restrict__ dst_idx, int64_t n, int64_t row_bytes)
{
    for (int64_t r = blockIdx.x; r < n; r += gridDim.x) {
        const char* a = src + src_idx[r] * ld_src;
        char* b = dst + dst_idx[r] * ld_dst;
        if (((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | row_bytes) & 15) == 0) {
            for (int64_t i = threadIdx.x; i < row_bytes / 16; i += blockDim.x)
                reinterpret_cast<uint4*>(b)[i] = reinterpret_cast<const uint4*>(a)[i];
        } else {
            for (int64_t i = threadIdx.x; i < row_bytes; i += blockDim.x) b[i] = a[i];
        }
    }
}

int floor_log2(int64_t v)
{
    int r = 0;
    while (v > 1) { v >>= 1; ++r; }
    return r;
}

// ------------------------------------------------------------ the cache
std::string cache_path()
{
    if (const char* e = getenv("RPYB_SIG_TUNE_CACHE")) return e;
    std::string base;
    if (const char* x = getenv("XDG_CACHE_HOME")) base = x;
    else if (const char* h = getenv("HOME")) base = std::string(h) + "/.cache";
    else base = "/tmp";
    return base + "/roughpy_b200/signature_schedules.json";
}

// The cache is a JSON object with one entry per line:
//   "key": {"g": 8, "wpb": 0, "seg": 0, "ms": 12.5},
std::map<std::string, Schedule> read_cache(const std::string& path)
{
    std::map<std::string, Schedule> out;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return out;
    char line[512];
    while (fgets(line, sizeof line, f)) {
        const char* q0 = strchr(line, '"');
        if (!q0) continue;
        const char* q1 = strchr(q0 + 1, '"');
        if (!q1) continue;
        Schedule sc;
        long long seg = 0;
        if (sscanf(q1 + 1, ": {\"g\": %d, \"wpb\": %d, \"seg\": %lld, \"ms\": %lf", &sc.g, &sc.wpb,
                   &seg, &sc.ms) == 4) {
            sc.seg = seg;
            sc.source = "cache";
            out[std::string(q0 + 1, q1)] = sc;
        }
    }
    fclose(f);
    return out;
}

void make_dirs(const std::string& path)
{
    for (size_t i = 1; i < path.size(); ++i) {
        if (path[i] == '/') {
            const std::string d = path.substr(0, i);
            mkdir(d.c_str(), 0755);
        }
    }
}

// Merges one entry into the cache file under an exclusive lock (processes
// tuning concurrently keep each other's entries).  Failures are ignored: the
// cache only saves tuning time.
void write_cache_entry(const std::string& path, const std::string& key, const Schedule& sc)
{
    make_dirs(path);
    const std::string lock_path = path + ".lock";
    const int lk = open(lock_path.c_str(), O_CREAT | O_RDWR, 0644);
    if (lk >= 0) flock(lk, LOCK_EX);
    auto entries = read_cache(path);
    entries[key] = sc;
    const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
    if (FILE* f = fopen(tmp.c_str(), "w")) {
        fprintf(f, "{\n");
        size_t i = 0;
        for (const auto& kv : entries) {
            fprintf(f, "\"%s\": {\"g\": %d, \"wpb\": %d, \"seg\": %lld, \"ms\": %.4f}%s\n",
                    kv.first.c_str(), kv.second.g, kv.second.wpb, (long long)kv.second.seg,
                    kv.second.ms, (++i < entries.size()) ? "," : "");
        }
        fprintf(f, "}\n");
        fclose(f);
        rename(tmp.c_str(), path.c_str());
    }
    if (lk >= 0) {
        flock(lk, LOCK_UN);
        close(lk);
    }
}

std::mutex& cache_mutex()
{
    static std::mutex m;
    return m;
}

// RPYB_SIG_SCHEDULE="g=8,wpb=0,seg=4096" (any subset; missing knobs default)
bool forced_schedule(Schedule& sc)
{
    const char* e = getenv("RPYB_SIG_SCHEDULE");
    if (!e || !*e) return false;
    std::string s(e);
    size_t pos = 0;
    while (pos < s.size()) {
        size_t comma = s.find(',', pos);
        if (comma == std::string::npos) comma = s.size();
        const std::string kv = s.substr(pos, comma - pos);
        const size_t eq = kv.find('=');
        if (eq != std::string::npos) {
            const std::string k = kv.substr(0, eq);
            const long long v = atoll(kv.c_str() + eq + 1);
            if (k == "g") sc.g = (int)v;
            else if (k == "wpb") sc.wpb = (int)v;
            else if (k == "seg") sc.seg = v;
        }
        pos = comma + 1;
    }
    sc.source = "forced";
    return true;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

struct rpyb_sig_plan {
    int mode = RPYB_F32;
    int width = 0, depth = 0;
    Geometry geo;
    int64_t n_streams = 0, total = 0, max_len = 0;
    std::vector<int64_t> offsets;          // host copy of the stream offsets
    bool specialised = false;
    Schedule sched;
    std::string key;
    int device = 0;

    // device layout of the current schedule
    DeviceBuf layout;                       // offsets, order, item tables, merge indices
    const int64_t* d_stream_offsets = nullptr;
    const int64_t* d_item_offsets = nullptr;
    const int64_t* d_order = nullptr;
    const int64_t* d_stream_order = nullptr; // longest-first order of whole streams
    const int64_t* d_dst = nullptr;         // nullptr when no stream is split
    int64_t n_items = 0;
    struct Level {
        int64_t n;
        const int64_t *out_idx, *lhs_idx, *rhs_idx;
    };
    std::vector<Level> levels;
    const int64_t* d_final_src = nullptr;
    const int64_t* d_final_dst = nullptr;
    int64_t n_final = 0;
    DeviceBuf rows;                         // segment and merge rows [n_rows, T]
    int64_t n_rows = 0;
    DeviceBuf queue;                        // work counter / generic-kernel workspace
    size_t queue_bytes = 0;
    // error report (allocated on first use)
    DeviceBuf ref_ws;
    size_t ref_bytes = 0;

    size_t elem() const { return mode == RPYB_F64 ? 8 : 4; }
};

namespace {

std::vector<int64_t> longest_first(const std::vector<int64_t>& off)
{
    const int64_t n = (int64_t)off.size() - 1;
    std::vector<int64_t> order(n);
    for (int64_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
        return off[x + 1] - off[x] > off[y + 1] - off[y];
    });
    return order;
}

int build_layout(rpyb_sig_plan* p, int64_t seg)
{
    const int64_t n = p->n_streams;
    const int64_t T = p->geo.size();
    // work items: whole streams, or the balanced segments of long ones
    std::vector<int64_t> item_off;
    std::vector<int64_t> dst;
    std::vector<std::vector<int64_t>> split_rows;   // per split stream: its segment rows
    std::vector<int64_t> split_stream;
    item_off.reserve(n + 1);
    item_off.push_back(0);
    int64_t nrows = 0;
    for (int64_t s = 0; s < n; ++s) {
        const int64_t a = p->offsets[s], len = p->offsets[s + 1] - a;
        const int64_t k = (seg > 0 && len > seg) ? (len + seg - 1) / seg : 1;
        if (k == 1) {
            item_off.push_back(p->offsets[s + 1]);
            dst.push_back(s);
            continue;
        }
        std::vector<int64_t> r;
        for (int64_t j = 1; j <= k; ++j) {
            item_off.push_back(a + (len * j) / k);
            dst.push_back(~nrows);
            r.push_back(nrows++);
        }
        split_rows.push_back(r);
        split_stream.push_back(s);
    }
    const int64_t n_items = (int64_t)dst.size();
    const std::vector<int64_t> order = longest_first(item_off);
    const std::vector<int64_t> stream_order = longest_first(p->offsets);
    // pairwise merge tree, level by level over all split streams
    std::vector<std::vector<int64_t>> lv_out, lv_lhs, lv_rhs;
    std::vector<int64_t> fin_src, fin_dst;
    {
        std::vector<std::vector<int64_t>> cur = split_rows;
        bool more = !cur.empty();
        while (more) {
            more = false;
            std::vector<int64_t> o, l, r;
            for (auto& rows : cur) {
                if (rows.size() < 2) continue;
                std::vector<int64_t> next;
                for (size_t i = 0; i + 1 < rows.size(); i += 2) {
                    l.push_back(rows[i]);
                    r.push_back(rows[i + 1]);
                    o.push_back(nrows);
                    next.push_back(nrows++);
                }
                if (rows.size() % 2) next.push_back(rows.back());
                rows = next;
                if (rows.size() > 1) more = true;
            }
            if (!o.empty()) {
                lv_out.push_back(o);
                lv_lhs.push_back(l);
                lv_rhs.push_back(r);
            }
        }
        for (size_t i = 0; i < cur.size(); ++i) {
            fin_src.push_back(cur[i][0]);
            fin_dst.push_back(split_stream[i]);
        }
    }
    // one device allocation for every table
    const bool any_split = !split_rows.empty();
    std::vector<int64_t> host;
    auto put = [&](const std::vector<int64_t>& v) {
        const size_t at = host.size();
        host.insert(host.end(), v.begin(), v.end());
        return at;
    };
    const size_t at_soff = put(p->offsets);
    const size_t at_ioff = put(item_off);
    const size_t at_order = put(order);
    const size_t at_sorder = put(stream_order);
    size_t at_dst = 0, at_fs = 0, at_fd = 0;
    if (any_split) {
        at_dst = put(dst);
        at_fs = put(fin_src);
        at_fd = put(fin_dst);
    }
    std::vector<size_t> at_lv;
    for (size_t i = 0; i < lv_out.size(); ++i) {
        at_lv.push_back(put(lv_out[i]));
        put(lv_lhs[i]);
        put(lv_rhs[i]);
    }
    int rc;
    if ((rc = p->layout.alloc(std::max<size_t>(host.size(), 1) * 8))) return rc;
    if (!host.empty())
        RPYB_CUDA(cudaMemcpy(p->layout.p, host.data(), host.size() * 8, cudaMemcpyHostToDevice));
    const int64_t* base = static_cast<const int64_t*>(p->layout.p);
    p->d_stream_offsets = base + at_soff;
    p->d_item_offsets = base + at_ioff;
    p->d_order = base + at_order;
    p->d_stream_order = base + at_sorder;
    p->n_items = n_items;
    p->d_dst = any_split ? base + at_dst : nullptr;
    p->d_final_src = any_split ? base + at_fs : nullptr;
    p->d_final_dst = any_split ? base + at_fd : nullptr;
    p->n_final = (int64_t)fin_src.size();
    p->levels.clear();
    for (size_t i = 0; i < lv_out.size(); ++i) {
        const int64_t m = (int64_t)lv_out[i].size();
        p->levels.push_back({m, base + at_lv[i], base + at_lv[i] + m, base + at_lv[i] + 2 * m});
    }
    p->n_rows = nrows;
    if ((rc = p->rows.alloc((size_t)nrows * (size_t)T * p->elem()))) return rc;
    return RPYB_OK;
}

int run_plan(rpyb_sig_plan* p, const void* inc, void* out, int64_t ld_out, cudaStream_t s)
{
    int rc;
    const int64_t T = p->geo.size();
    if (!p->specialised) {
        return rpyb_signature(p->mode, p->width, p->depth, p->n_streams, p->d_stream_offsets, inc,
                              out, ld_out, p->d_stream_order, p->queue.p, p->queue_bytes, s);
    }
    if ((rc = signature_launch(p->mode, p->width, p->depth, p->sched.g, p->sched.wpb, p->n_items,
                               p->d_item_offsets, inc, out, ld_out, p->d_order, p->d_dst,
                               p->rows.p, T, static_cast<int*>(p->queue.p), s)))
        return rc;
    for (const auto& lv : p->levels) {
        if ((rc = rpyb_ft_mul_gather(p->mode, p->width, p->depth, lv.n, p->rows.p, p->rows.p,
                                     p->rows.p, T, lv.out_idx, lv.lhs_idx, lv.rhs_idx, 0, s)))
            return rc;
    }
    if (p->n_final > 0) {
        const int64_t blocks = std::min<int64_t>(p->n_final, 4096);
        copy_rows_kernel<<<(unsigned)blocks, 256, 0, s>>>(
            static_cast<const char*>(p->rows.p), T * (int64_t)p->elem(), static_cast<char*>(out),
            ld_out * (int64_t)p->elem(), p->d_final_src, p->d_final_dst, p->n_final,
            T * (int64_t)p->elem());
        RPYB_CUDA(cudaGetLastError());
    }
    return RPYB_OK;
}

std::vector<Schedule> candidates(const rpyb_sig_plan* p)
{
    std::vector<Schedule> out;
    int gs[4], count = 0;
    signature_lane_shapes(p->mode, p->width, p->depth, gs, &count);
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<int64_t> segs = {0};
    // split only when the whole streams leave the GPU short of work: fewer
    // warp items than a few waves of resident warps
    const int64_t lanes = signature_lanes_per_stream(p->mode, p->width, p->depth, gs[0]);
    const int64_t warp_items = p->n_streams * ((lanes + 31) / 32);
    if (warp_items < (int64_t)sms * 8 * 4) {
        for (int64_t L : {256, 1024, 4096, 16384})
            if (2 * L <= p->max_len) segs.push_back(L);
    }
    for (int i = 0; i < count; ++i)
        for (int wpb : {0, 4})
            for (int64_t seg : segs) {
                Schedule sc;
                sc.g = gs[i];
                sc.wpb = wpb;
                sc.seg = seg;
                sc.source = "tuned";
                out.push_back(sc);
            }
    return out;
}

int tune(rpyb_sig_plan* p, cudaStream_t s)
{
    int rc;
    const int64_t T = p->geo.size();
    DeviceBuf inc, out;
    const int64_t nval = std::max<int64_t>(p->total * p->width, 1);
    if ((rc = inc.alloc((size_t)nval * p->elem()))) return rc;
    if ((rc = out.alloc((size_t)p->n_streams * (size_t)T * p->elem()))) return rc;
    const double mean_len = std::max(1.0, (double)p->total / std::max<int64_t>(p->n_streams, 1));
    synthetic_rows_kernel<<<1024, 256, 0, s>>>(inc.p, nval, p->mode == RPYB_F64,
                                               std::sqrt(3.0 / mean_len));
    RPYB_CUDA(cudaGetLastError());
    cudaEvent_t e0, e1;
    RPYB_CUDA(cudaEventCreate(&e0));
    RPYB_CUDA(cudaEventCreate(&e1));
    Schedule best;
    double best_ms = 1e300;
    for (Schedule sc : candidates(p)) {
        if ((rc = build_layout(p, sc.seg))) break;
        p->sched = sc;
        if ((rc = run_plan(p, inc.p, out.p, T, s))) break;   // warm-up
        double ms_min = 1e300;
        for (int r = 0; r < 2 && rc == RPYB_OK; ++r) {
            cudaEventRecord(e0, s);
            rc = run_plan(p, inc.p, out.p, T, s);
            cudaEventRecord(e1, s);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(RPYB_E_CUDA, "tuning run failed");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_min = std::min(ms_min, (double)ms);
        }
        if (rc) break;
        if (ms_min < best_ms) {
            best_ms = ms_min;
            best = sc;
            best.ms = ms_min;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    p->sched = best;
    return RPYB_OK;
}

}  // namespace

extern "C" {

RPYB_API int rpyb_sig_plan_create(int mode, int32_t width, int32_t depth, int64_t n_streams,
                                  const int64_t* offsets_host, int32_t flags, void* stream,
                                  rpyb_sig_plan** out)
{
    int rc;
    if (!out) return fail(RPYB_E_INVALID, "null plan pointer");
    *out = nullptr;
    if (mode != RPYB_F32 && mode != RPYB_F64) return fail(RPYB_E_INVALID, "unsupported mode");
    Geometry g;
    if ((rc = make_geometry(width, depth, g))) return rc;
    if (n_streams < 0) return fail(RPYB_E_INVALID, "negative number of streams");
    if (!offsets_host) return fail(RPYB_E_INVALID, "null offsets");
    if (offsets_host[0] != 0) return fail(RPYB_E_INVALID, "offsets must start at 0");
    int64_t max_len = 0;
    for (int64_t i = 0; i < n_streams; ++i) {
        const int64_t len = offsets_host[i + 1] - offsets_host[i];
        if (len < 0) return fail(RPYB_E_INVALID, "offsets must be non-decreasing");
        max_len = std::max(max_len, len);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto* p = new rpyb_sig_plan();
    p->mode = mode;
    p->width = width;
    p->depth = depth;
    p->geo = g;
    p->n_streams = n_streams;
    p->total = offsets_host[n_streams];
    p->max_len = max_len;
    p->offsets.assign(offsets_host, offsets_host + n_streams + 1);
    cudaGetDevice(&p->device);
    int gs[4], count = 0;
    p->specialised = signature_lane_shapes(mode, width, depth, gs, &count);
    p->queue_bytes = (size_t)std::max<int64_t>(
        256, rpyb_signature_workspace_size(mode, width, depth, n_streams));
    if ((rc = p->queue.alloc(p->queue_bytes))) {
        delete p;
        return rc;
    }
    if (p->specialised && n_streams > 0) {
        cudaDeviceProp prop;
        std::string dev_name = "gpu";
        if (cudaGetDeviceProperties(&prop, p->device) == cudaSuccess) dev_name = prop.name;
        for (char& c : dev_name)
            if (c == ' ' || c == '"') c = '_';
        p->key = dev_name + "|" + (mode == RPYB_F64 ? "f64" : "f32") + "|w" +
                 std::to_string(width) + "d" + std::to_string(depth) + "|L" +
                 std::to_string(floor_log2(std::max<int64_t>(max_len, 1))) + "|n" +
                 std::to_string(floor_log2(n_streams));
        Schedule sc;
        bool have = forced_schedule(sc);
        const std::string path = cache_path();
        if (!have) {
            std::lock_guard<std::mutex> lk(cache_mutex());
            auto entries = read_cache(path);
            auto it = entries.find(p->key);
            if (it != entries.end()) {
                sc = it->second;
                have = true;
            }
        }
        if (have) {
            // a cached or forced lane shape must exist for this mode and shape
            bool ok = sc.g == 0;
            for (int i = 0; i < count; ++i) ok = ok || gs[i] == sc.g;
            if (!ok) sc.g = 0;
            p->sched = sc;
        } else if (flags & RPYB_SIG_PLAN_TUNE) {
            if ((rc = tune(p, s))) {
                delete p;
                return rc;
            }
            std::lock_guard<std::mutex> lk(cache_mutex());
            write_cache_entry(path, p->key, p->sched);
        }
    }
    if ((rc = build_layout(p, p->specialised ? p->sched.seg : 0))) {
        delete p;
        return rc;
    }
    *out = p;
    return RPYB_OK;
}

RPYB_API int rpyb_sig_plan_run(rpyb_sig_plan* p, const void* increments, void* out, int64_t ld_out,
                               double* err_out, void* stream)
{
    int rc;
    if (!p) return fail(RPYB_E_INVALID, "null plan");
    if (p->n_streams == 0) return RPYB_OK;
    if (!out) return fail(RPYB_E_INVALID, "null output");
    if (p->n_streams > 1 && ld_out < p->geo.size()) return fail(RPYB_E_INVALID, "ld_out too small");
    if (p->total > 0 && !increments) return fail(RPYB_E_INVALID, "null increments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // with no rows the kernels read no increment; any aligned pointer will do
    const void* inc = p->total > 0 ? increments : p->queue.p;
    if ((rc = run_plan(p, inc, out, ld_out, s))) return rc;
    if (!err_out) return RPYB_OK;
    if (p->mode == RPYB_F64) {
        RPYB_CUDA(cudaMemsetAsync(err_out, 0, (size_t)p->n_streams * sizeof(double), s));
        return RPYB_OK;
    }
    // the float64 path on the same increments, then the per-level comparison
    const size_t need = (size_t)rpyb_signature_batched_workspace_size(
        p->mode, p->width, p->depth, p->n_streams, p->total, 1);
    if (p->ref_bytes < need) {
        RPYB_CUDA(cudaStreamSynchronize(s));
        if ((rc = p->ref_ws.alloc(need))) return rc;
        p->ref_bytes = need;
    }
    return signature_error_report(p->width, p->depth, p->n_streams, p->d_stream_offsets, inc,
                                  p->total, out, ld_out, p->d_stream_order, err_out, p->ref_ws.p,
                                  p->ref_bytes, s);
}

RPYB_API int rpyb_sig_plan_describe(const rpyb_sig_plan* p, char* buf, int64_t cap)
{
    if (!p) return fail(RPYB_E_INVALID, "null plan");
    char tmp[512];
    const int n = snprintf(
        tmp, sizeof tmp,
        "{\"key\": \"%s\", \"kernel\": \"%s\", \"g\": %d, \"wpb\": %d, \"seg\": %lld, "
        "\"items\": %lld, \"merge_levels\": %d, \"source\": \"%s\", \"ms\": %.4f}",
        p->key.c_str(), p->specialised ? "specialised" : "generic", p->sched.g, p->sched.wpb,
        (long long)p->sched.seg, (long long)p->n_items, (int)p->levels.size(),
        p->sched.source.c_str(), p->sched.ms);
    if (buf && cap > 0) {
        strncpy(buf, tmp, (size_t)cap - 1);
        buf[cap - 1] = '\0';
    }
    return n;
}

RPYB_API int rpyb_sig_plan_free(rpyb_sig_plan* p)
{
    delete p;
    return RPYB_OK;
}

}  // extern "C"
