"""Benchmark of the B200 tensor-algebra hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Headline workload (one "step" = one pass over one batch):
  uneven batched signatures -- 4096 streams per GPU, lengths uniform in
  [16, 4096] (seeded), width 8, depth 5, Brownian increments N(0, 1/len),
  float32 storage with compensated accumulation, one persistent launch.
The line also carries the float64 path on the same inputs (speed and the
max per-level relative error of the float32 path against it) and the
free-tensor FMA sweep (1024 pairs, (d,N) in {(2,12),(4,8),(6,6),(8,6)},
float64 and float32) as % of the measured HBM bandwidth.

Multi-GPU (torchrun): every rank computes its own 4096 streams (weak
scaling); no collective touches the data path; times are the max over ranks.
``--impl reference`` times RoughPy's own CPU implementation of the path
(the reference roughpy.compute extension built from its sources, chaining
ft_fmexp per stream) on a bounded sample per step, using every host core.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import pathlib
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = ("sig streams/s FP32-comp vs FP64 at ≤1e-6 rel err; "
          "tensor-mul % of HBM peak")
WIDTH, DEPTH = 8, 5
N_STREAMS = 4096
LEN_LO, LEN_HI = 16, 4096
FMA_PER_STEP = 42792          # Horner Chen step at (8,5): sum_k sum_{i<=k} 8^i
SWEEP = [(2, 12), (4, 8), (6, 6), (8, 6)]
SWEEP_BATCH = 1024
E2E_CHUNKS = 16
SM_COUNT_B200 = 148
FP32_LANES_PER_SM = 128
# DRAM bytes (read + write) per stream of the float32 signature kernel on this
# workload: 68.1 + 98.2 MB measured by ncu on the 1024-stream slice
# (`bench.py --profile-slice 1024`, profiles/signature_w8d5_f32c_f64.md); the
# traffic is inputs plus outputs, so it scales with the number of streams.
SIG_TRAFFIC_BYTES_PER_STREAM = (68.1e6 + 98.2e6) / 1024


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(seed: int, n: int = N_STREAMS):
    rng = np.random.default_rng(seed)
    lens = rng.integers(LEN_LO, LEN_HI + 1, size=n)
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    inc = np.empty((int(off[-1]), WIDTH), dtype=np.float32)
    for s in range(n):
        L = int(lens[s])
        inc[off[s]:off[s + 1]] = rng.normal(0.0, np.sqrt(1.0 / L), size=(L, WIDTH))
    return lens, off, inc


def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ------------------------------------------------------------- CPU baseline
def _cpu_worker(args):
    """Reference CPU path for a list of streams: chained ft_fmexp (float64)."""
    kind, width, depth, chunks = args
    import oracle
    if kind == "reference":
        rpc = oracle.ref_compute()
        basis = rpc.TensorBasis(width, depth)
        for inc in chunks:
            sig = np.zeros(basis.size())
            sig[0] = 1.0
            x = np.zeros(basis.size())
            for row in inc:
                x[1:1 + width] = row
                sig = rpc.ft_fmexp(rpc.FreeTensor(sig, basis), rpc.FreeTensor(x, basis)).data
    else:
        for inc in chunks:
            oracle.signature(width, depth, inc)
    return len(chunks)


def cpu_kind():
    import oracle
    return "reference" if oracle.ref_compute() is not None else "port"


class CpuBaseline:
    """Times the reference CPU path on all host cores (spawned workers)."""

    def __init__(self, cores: int | None = None):
        self.cores = cores or len(os.sched_getaffinity(0))
        self.kind = cpu_kind()
        ctx = mp.get_context("spawn")
        self.pool = ctx.Pool(self.cores)
        # warm the workers (imports, reference module load)
        self.pool.map(_cpu_worker, [(self.kind, WIDTH, DEPTH, [])] * self.cores)

    def run(self, streams):
        parts = [streams[i::self.cores] for i in range(self.cores)]
        t0 = time.perf_counter()
        done = sum(self.pool.map(_cpu_worker, [(self.kind, WIDTH, DEPTH, p) for p in parts]))
        return done, time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def sample_streams(inc, off, idx):
    return [np.ascontiguousarray(inc[off[s]:off[s + 1]], dtype=np.float64) for s in idx]


# ------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            return None
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm, mx = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            sms.append(sm)
            maxs.append(mx)
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sms:
            return None
        return {"sm_mhz": float(np.median(sms)), "sm_max_mhz": float(max(maxs)),
                "reasons": sorted(reasons), "samples": len(sms)}


# ------------------------------------------------------------- ranks
def rank_workload(rank, world, scaling):
    """This rank's streams: (lens, off, inc, shard).

    weak: its own 4096-stream batch (seed 2 + rank), shard = (0, 4096);
    strong: its length-balanced contiguous slice (roughpy_b200.distributed.
    shard_bounds) of the one 4096-stream batch (seed 2), shard = (lo, hi)."""
    if scaling == "weak":
        lens, off, inc = make_workload(seed=2 + rank)
        return lens, off, inc, (0, N_STREAMS)
    from roughpy_b200.distributed import shard_bounds
    lens, off, inc = make_workload(seed=2)
    lo, hi = shard_bounds(off, world)[rank]
    local_off = off[lo:hi + 1] - off[lo]
    return lens[lo:hi], local_off, inc[off[lo]:off[hi]], (int(lo), int(hi))


def global_streams(world, scaling):
    return world * N_STREAMS if scaling == "weak" else N_STREAMS


def dry_run(args, rank, world):
    """The rank plumbing without a GPU: process group (gloo), per-rank
    workload and shard, barriers, max-over-ranks timing and the JSON line.
    The timed step is a host copy of the rank's increment rows, so the
    number measures nothing but the plumbing; the line says so."""
    import torch
    import torch.distributed as dist
    lens, off, inc, shard = rank_workload(rank, world, args.scaling)
    buf = np.empty_like(inc)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        np.copyto(buf, inc)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        np.copyto(buf, inc)
    if world > 1:
        dist.barrier()
    ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps)
    shards = [None] * world
    if world > 1:
        dist.all_gather_object(shards, shard)
    else:
        shards = [shard]
    if rank != 0:
        return None
    return {"metric": METRIC, "value": round(global_streams(world, args.scaling) / (ms / 1e3), 1),
            "unit": "streams/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": args.scaling,
            "vs_baseline": None, "dtype": "none (dry run)", "data": "synthetic",
            "dry_run": True,
            "config": {"workload": "rank plumbing only: the step copies the rank's rows on "
                                   "the host", "global_batch": global_streams(world, args.scaling),
                       "shards": shards}}


# ------------------------------------------------------------- GPU arm
def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from roughpy_b200 import signatures as S

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lens, off, inc, shard = rank_workload(rank, world, args.scaling)
    n_local = int(len(lens))
    T = S.tensor_size(WIDTH, DEPTH)
    inc_d = torch.from_numpy(inc).to(dev)
    plan = S.SignaturePlan(off, WIDTH, DEPTH, "f32c", device=dev)
    out_d = torch.empty((n_local, T), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    n_global = global_streams(world, args.scaling)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident timing (value)
    for _ in range(args.warmup):
        plan.run(inc_d, out_d)
    barrier()
    clocks = ClockSampler(local_rank) if rank == 0 else None
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        plan.run(inc_d, out_d)
    ev1.record(stream)
    barrier()
    ms_total = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = ms_total / args.steps
    value = n_global / (ms_step / 1e3)

    # ---- end to end through the C ABI (rpyb_signature_host) from pinned host
    # buffers: host->device copies, kernels and device->host copies, chunked
    # so that the transfers overlap the computation
    inc_h = torch.from_numpy(inc).pin_memory()
    out_h = torch.empty((n_local, T), dtype=torch.float32).pin_memory()
    for _ in range(args.warmup):
        plan.run_host_pipelined(inc_h, out_h, n_chunks=E2E_CHUNKS)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.run_host_pipelined(inc_h, out_h, n_chunks=E2E_CHUNKS)
    e1.record(stream)
    barrier()
    clk = clocks.stop() if clocks else None
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    e2e_value = n_global / (e2e_ms / 1e3)

    # ---- float64 path on the same inputs: speed and the accuracy of float32
    plan64 = S.SignaturePlan(off, WIDTH, DEPTH, "f64", device=dev)
    inc64 = inc_d.double()
    out64 = torch.empty((n_local, T), dtype=torch.float64, device=dev)
    for _ in range(max(1, args.warmup // 2)):
        plan64.run(inc64, out64)
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    k64 = max(1, min(args.steps, 5))
    f0.record(stream)
    for _ in range(k64):
        plan64.run(inc64, out64)
    f1.record(stream)
    barrier()
    ms64 = max_over_ranks(f0.elapsed_time(f1)) / k64
    _, err_rows = plan.run(inc_d, out_d, report_error=True)
    torch.cuda.synchronize(dev)
    err = max_over_ranks(level_rel_err_torch(out_d, out64, WIDTH, DEPTH))
    err_report = max_over_ranks(float(err_rows.max()))
    del inc64, out64

    result = None
    if rank == 0:
        pk, pk_kind = peaks()
        sm_mhz = (clk or {}).get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
        fp32_peak = 2 * FP32_LANES_PER_SM * SM_COUNT_B200 * sm_mhz * 1e6 / 1e12
        algo_flops = 2.0 * FMA_PER_STEP * float(lens.sum())
        achieved = algo_flops / (ms_step / 1e3) / 1e12   # this GPU's launch
        traffic = SIG_TRAFFIC_BYTES_PER_STREAM * n_local if SIG_TRAFFIC_BYTES_PER_STREAM else None
        sweep = fma_sweep(dev, pk["hbm_gbs"]) if not args.no_sweep else None
        result = {
            "metric": METRIC,
            "value": round(value, 1),
            "unit": "streams/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_step, 4),
            "higher_is_better": True,
            "scaling": args.scaling,
            "vs_baseline": None,
            "dtype": "f32 (compensated)",
            "data": "synthetic (seeded Brownian increments)",
            "config": {
                "workload": "uneven batched signatures: 4096 streams "
                            f"{'per GPU' if args.scaling == 'weak' else 'in all'}, lengths "
                            "U{16..4096}, width 8, depth 5, increments N(0,1/len), FP32-comp",
                "global_batch": n_global,
                "width": WIDTH, "depth": DEPTH,
                "parallelism": f"dp{world} (streams sharded, no collective)",
                "shard": list(shard),
                "schedule": plan.schedule(),
                "l2": "inputs+outputs 0.9 GB per step > 126 MB L2 (no flush needed)",
            },
            "f64_path": {"value": round(n_global / (ms64 / 1e3), 1),
                         "unit": "streams/s", "ms_per_step": round(ms64, 4),
                         "schedule": plan64.schedule()},
            "f32c_speedup_vs_f64": round(ms64 / ms_step, 3),
            "max_rel_err_vs_f64": err,
            "max_rel_err_reported": err_report,
            "roofline": {
                "bound": "fp32_fma", "achieved": round(achieved, 3), "peak": round(fp32_peak, 2),
                "unit": "TFLOP/s", "frac": round(achieved / fp32_peak, 4),
                "traffic": traffic,
                "traffic_unit": "bytes per launch (ncu dram read+write, 1024-stream "
                                "capture scaled by the stream count)",
                "note": "algorithmic 2*42792 flop per increment; FP32 CUDA-core peak "
                        "= 148 SM x 128 lanes x 2 x sampled SM clock (computed: no FP32 figure "
                        "is measured); the float32 kernel also runs its low levels on the "
                        "FP64 pipe",
            },
            "tensor_mul": sweep,
            "e2e": {"value": round(e2e_value, 1), "unit": "streams/s",
                    "h2d_bytes_per_step": int(inc.nbytes),
                    "d2h_bytes_per_step": int(n_local * T * 4),
                    "ms_per_step": round(e2e_ms, 4),
                    "path": f"rpyb_signature_host, pinned host buffers, {E2E_CHUNKS} chunks "
                            "with copies overlapping kernels"},
            "gpu_launches": args.steps,
            "clocks": clk,
            "peaks_source": pk_kind,
        }
    return result, (lens, off, inc)


def level_rel_err_torch(got, want, width, depth):
    import torch
    db = [0]
    for _ in range(depth + 1):
        db.append(1 + width * db[-1])
    worst = 0.0
    g = got.double()
    for k in range(depth + 1):
        a = g[:, db[k]:db[k + 1]]
        b = want[:, db[k]:db[k + 1]]
        num = (a - b).abs().amax(dim=1)
        den = b.abs().amax(dim=1)
        rel = torch.where(den > 0, num / torch.where(den > 0, den, torch.ones_like(den)), num)
        worst = max(worst, float(rel.max()))
    return worst


_FLUSH = {}


def flush_l2(torch, dev):
    """Evict L2 (126 MB): write a 256 MB buffer, then read it back so that
    the lines left in L2 are clean and no write-back falls in the next timed
    launch."""
    buf = _FLUSH.get(str(dev))
    if buf is None:
        buf = _FLUSH[str(dev)] = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    buf.fill_(1.0)
    buf.sum()


def fma_sweep(dev, hbm_gbs):
    """Config-2 FMA sweep: C += A (x) B over 1024 pairs; GB/s vs HBM."""
    import torch
    from roughpy_b200 import _lib
    res = {}
    stream = torch.cuda.current_stream(dev).cuda_stream
    for (w, d) in SWEEP:
        T = int(_lib.lib.rpyb_tensor_size(w, d))
        for dt, code, es, name in ((torch.float64, _lib.F64, 8, "f64"),
                                   (torch.float32, _lib.F32, 4, "f32c")):
            g = torch.Generator(device=dev).manual_seed(1)
            A = torch.randn(SWEEP_BATCH, T, dtype=dt, device=dev, generator=g)
            B = torch.randn(SWEEP_BATCH, T, dtype=dt, device=dev, generator=g)
            C = torch.randn(SWEEP_BATCH, T, dtype=dt, device=dev, generator=g)

            def run():
                _lib.check(_lib.lib.rpyb_ft_fma(code, w, d, SWEEP_BATCH, C.data_ptr(),
                                                A.data_ptr(), B.data_ptr(), T, T, T, None,
                                                stream))
            for _ in range(3):
                run()
            torch.cuda.synchronize(dev)
            # each launch timed alone after an L2 flush (the (2,12) float32
            # operands, 100 MB, would otherwise stay resident in the 126 MB L2)
            reps = 10
            ms = 0.0
            for _ in range(reps):
                flush_l2(torch, dev)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                run()
                e1.record()
                torch.cuda.synchronize(dev)
                ms += e0.elapsed_time(e1) / reps
            gbs = 4.0 * T * es * SWEEP_BATCH / (ms / 1e3) / 1e9
            res[f"w{w}d{d}_{name}"] = {"ms": round(ms, 4), "GB/s": round(gbs, 1),
                                       "frac_hbm": round(gbs / hbm_gbs, 3)}
            del A, B, C
    torch.cuda.empty_cache()
    res["timing"] = "each launch timed alone by CUDA events after an L2 flush; mean of 10"
    return res


# ------------------------------------------------------------- other workloads
def _events_time(torch, fn, reps, warm=2):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def plain_f64_signatures(dev):
    """256 streams x 128 increments, width 4, depth 5, float64 (the reference's
    CPU-runnable case), with the reference timed on one core beside it."""
    import torch
    from roughpy_b200 import signatures as S
    import oracle
    rng = np.random.default_rng(0)
    n, L, w, d = 256, 128, 4, 5
    inc = rng.normal(0, np.sqrt(1.0 / 128), size=(n * L, w))
    off = np.arange(n + 1, dtype=np.int64) * L
    plan = S.SignaturePlan(off, w, d, "f64", device=dev)
    x = torch.from_numpy(inc).to(dev)
    out = torch.empty((n, plan.size), dtype=torch.float64, device=dev)
    ms = _events_time(torch, lambda: plan.run(x, out), 50)
    got = out.cpu().numpy()
    want = oracle.signatures(w, d, inc[:16 * L], off[:17])
    err = float(np.max(np.abs(got[:16] - want)) / np.max(np.abs(want)))
    # the same launch replayed from a CUDA graph (no per-call launch overhead)
    graph, gout = plan.capture(x)
    ms_graph = _events_time(torch, graph.replay, 50)
    graph_same = bool(torch.equal(gout, out))
    del graph
    ref = {}
    rpc = oracle.ref_compute()
    if rpc is not None:
        t0 = time.perf_counter()
        _cpu_worker(("reference", w, d, [inc[s * L:(s + 1) * L] for s in range(32)]))
        dt = time.perf_counter() - t0
        ref = {"value": round(32 / dt, 1), "unit": "streams/s", "cores": 1, "kind": "reference",
               "sample": "32 of the 256 streams, chained roughpy.compute ft_fmexp"}
    return {"workload": "256 streams x 128 increments, width 4, depth 5, float64",
            "value": round(n / (ms / 1e3), 1), "unit": "streams/s", "ms": round(ms, 4),
            "cuda_graph": {"value": round(n / (ms_graph / 1e3), 1), "ms": round(ms_graph, 4),
                           "same_output": graph_same},
            "max_rel_err_vs_oracle": err, "cpu_reference_1_core": ref}


def long_streams(dev):
    """A few long streams: 8 streams of 2^17 increments, width 8, depth 5,
    float32 compensated.  Whole streams leave most of the GPU idle (16 warps
    each); the tuned plan cuts them into time segments merged by Chen
    products.  Both schedules are timed on the same inputs."""
    import torch
    from roughpy_b200 import signatures as S
    n, L = 8, 1 << 17
    rng = np.random.default_rng(6)
    inc = rng.normal(0, np.sqrt(1.0 / L), size=(n * L, WIDTH)).astype(np.float32)
    off = np.arange(n + 1, dtype=np.int64) * L
    x = torch.from_numpy(inc).to(dev)
    out = torch.empty((n, S.tensor_size(WIDTH, DEPTH)), dtype=torch.float32, device=dev)
    res = {"workload": "8 streams x 2^17 increments, width 8, depth 5, float32 compensated"}
    old = os.environ.get("RPYB_SIG_SCHEDULE")
    try:
        os.environ["RPYB_SIG_SCHEDULE"] = "seg=0"
        whole = S.SignaturePlan(off, WIDTH, DEPTH, "f32c", device=dev)
    finally:
        if old is None:
            os.environ.pop("RPYB_SIG_SCHEDULE", None)
        else:
            os.environ["RPYB_SIG_SCHEDULE"] = old
    tuned = S.SignaturePlan(off, WIDTH, DEPTH, "f32c", device=dev, tune=True)
    for name, plan in (("whole_streams", whole), ("tuned", tuned)):
        ms = _events_time(torch, lambda: plan.run(x, out), 3, warm=2)
        res[name] = {"ms": round(ms, 3), "value": round(n / (ms / 1e3), 1), "unit": "streams/s",
                     "schedule": plan.schedule()}
    _, err = tuned.run(x, out, report_error=True)
    res["tuned_max_rel_err_vs_f64"] = float(err.max())
    res["speedup_tuned_vs_whole"] = round(res["whole_streams"]["ms"] / res["tuned"]["ms"], 2)
    return res


def dyadic_queries(dev):
    """Dyadic-cache stream queries: 2^16 events at t_i = i 2^-16, width 6,
    depth 5, resolution 16, 100000 clopen queries with endpoints on the 2^-16
    grid; log-signatures (Chen reduction over cached dyadic nodes through the
    tree's range-product table, float64 log and Hall projection).  The tree
    and the table are built (and timed, as a process's second build) before
    the queries.  The reference's uncached recursion is estimated
    from its timed two-element CBH times the exact number it would perform."""
    import torch
    from roughpy_b200.streams import LieIncrementStream
    n = 1 << 16
    rng = np.random.default_rng(3)
    inc = rng.normal(0, np.sqrt(1.0 / n), size=(n, 6))
    idx = np.arange(n) / n
    nq = 100000
    q = np.sort(np.floor(rng.uniform(0, 1, size=(nq, 2)) * n) / n, axis=1)
    res = {"workload": "2^16 events, width 6, depth 5, resolution 16, 100000 queries"}
    lies = {}
    for mode, data in (("f32c", inc.astype(np.float32)),
                       ("f64", inc.astype(np.float32).astype(np.float64))):
        # warm-up on a small stream of the same shape: first-use costs (kernel
        # module loading, Lie map upload, scratch pool growth) stay untimed
        warm = LieIncrementStream.from_increments(data[:256], indices=idx[:256], width=6,
                                                  depth=5, resolution=16, device=dev)
        warm.log_signature_batch(q[:1000, 0] / 256, q[:1000, 1] / 256)
        del warm
        # the first full-size build of a process also pays first-use costs
        # (measured 12-56 ms against 11-13 ms for later builds): built once
        # untimed-in-the-value, then rebuilt and timed
        first = {}
        for attempt in range(2):
            st = LieIncrementStream.from_increments(data, indices=idx, width=6, depth=5,
                                                    resolution=16, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st._build_tree()
            torch.cuda.synchronize()
            tb = time.perf_counter() - t0
            t0 = time.perf_counter()
            st.build_range_table()
            torch.cuda.synchronize()
            tt = time.perf_counter() - t0
            if attempt == 0:
                first = {"tree_build_ms": round(tb * 1e3, 2), "range_table_ms": round(tt * 1e3, 2)}
                del st
                torch.cuda.empty_cache()
        st.log_signature_batch(q[:, 0], q[:, 1])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lie = st.log_signature_batch(q[:, 0], q[:, 1])
        torch.cuda.synchronize()
        tq = time.perf_counter() - t0
        lies[mode] = lie.cpu().numpy()
        res[mode] = {"tree_build_ms": round(tb * 1e3, 2), "range_table_ms": round(tt * 1e3, 2),
                     "first_build": first, "queries_s": round(tq, 4),
                     "value": round(nq / tq, 1), "unit": "queries/s (wall clock, host "
                                                         "dissection included)"}
        del st
        torch.cuda.empty_cache()
    scale = np.maximum(np.abs(lies["f64"]).max(axis=1, keepdims=True), 1e-300)
    res["f32c_max_rel_err_vs_f64"] = float((np.abs(lies["f32c"] - lies["f64"]) / scale).max())
    res["cpu_reference_estimate"] = _dyadic_reference_estimate(q)
    return res


def _dyadic_reference_estimate(q):
    import oracle
    rpc = oracle.ref_compute()
    if rpc is None:
        return None
    from roughpy_b200.streams import _dissect_batch
    R = 16
    tols = np.full(q.shape[0], 0, dtype=np.int32)
    for i, (a, b) in enumerate(q):
        L = b - a
        tols[i] = R if L == 0 else max(R, (-min(0, np.frexp(L)[1] - 1)) + 2)
    k, p, off = _dissect_batch(q[:, 0], q[:, 1], tols)
    # a piece of power p < R recurses to 2^(R-p) cached leaves and performs
    # 2^(R-p) - 1 two-element CBHs; each query adds one final CBH
    cbh2 = int(np.sum(np.where(p < R, (np.int64(1) << np.maximum(R - p, 0)) - 1, 0)))
    finals = int(np.sum(np.diff(off) > 1))
    tb = rpc.TensorBasis(6, 5)
    lb = rpc.LieBasis(6, 5)
    rng = np.random.default_rng(0)
    a = rng.normal(0, 1e-2, size=lb.size())
    b = rng.normal(0, 1e-2, size=lb.size())
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        ta = rpc.lie_to_tensor(rpc.Lie(a, lb), tb)
        tbb = rpc.lie_to_tensor(rpc.Lie(b, lb), tb)
        x = rpc.ft_fmexp(rpc.ft_exp(ta), tbb)
        rpc.tensor_to_lie(rpc.ft_log(x), lb)
    per = (time.perf_counter() - t0) / reps
    est = (cbh2 + finals) * per
    return {"value": round(q.shape[0] / est, 6), "unit": "queries/s (estimated)",
            "cores": 1, "kind": "reference",
            "model": f"{cbh2 + finals} two-element CBHs for the 100000 queries x "
                     f"{per * 1e3:.3f} ms measured per reference CBH at (6,5)",
            "estimated_seconds": round(est, 1)}


def signature_backward(dev):
    """512 streams x 1024 increments, width 5, depth 6, loss <W, sig>; forward
    by the signature kernel, backward by the adjoint kernel (checkpoint 64)."""
    import torch
    from roughpy_b200 import signatures as S
    n, L, w, d = 512, 1024, 5, 6
    rng = np.random.default_rng(4)
    inc = rng.normal(0, np.sqrt(1.0 / L), size=(n * L, w))
    off = np.arange(n + 1, dtype=np.int64) * L
    T = S.tensor_size(w, d)
    W = torch.from_numpy(rng.normal(size=(T,))).to(dev)
    res = {"workload": "512 x 1024 increments, width 5, depth 6, loss <W, sig>"}
    grads = {}
    for mode, dt in (("f32c", torch.float32), ("f64", torch.float64)):
        plan = S.SignaturePlan(off, w, d, mode, device=dev)
        x0 = torch.from_numpy(inc).to(dev, dt)

        def step():
            x = x0.clone().requires_grad_(True)
            sig = S.signature_with_grad(x, plan)
            (sig.double() * W).sum().backward()
            return x.grad
        ms = _events_time(torch, step, 3, warm=1)
        grads[mode] = step().double()
        res[mode] = {"ms_forward_backward": round(ms, 3),
                     "value": round(n / (ms / 1e3), 1), "unit": "streams/s"}
    g64 = grads["f64"]
    res["f32c_grad_max_rel_err_vs_f64"] = float((grads["f32c"] - g64).abs().max() /
                                                g64.abs().max())
    # the adjoint kernel alone (one launch over all streams)
    for mode, dt in (("f32c", torch.float32), ("f64", torch.float64)):
        launch = _backward_launch(mode, dt, n, L, w, d, inc, W, dev)
        res[mode]["ms_backward_kernel"] = round(_events_time(torch, launch, 3, warm=1), 3)
    # roofline of the adjoint kernel: a forward recomputation plus the two
    # adjoint products (with respect to the state and to the increment), each
    # of the forward's 24,405 FMA per increment at (5,6), all accumulated in
    # float64 on the FP64 pipe (148 SMs x 64 lanes x 2 flop x clock)
    fma_per_inc = 24405
    flops = 2.0 * 3 * fma_per_inc * n * L
    fp64_peak = 148 * 64 * 2 * 1965e6 / 1e12
    ms = res["f32c"]["ms_backward_kernel"]
    ach = flops / (ms / 1e3) / 1e12
    res["roofline"] = {"bound": "fp64_fma", "achieved": round(ach, 3), "peak": round(fp64_peak, 2),
                       "unit": "TFLOP/s", "frac": round(ach / fp64_peak, 4),
                       "note": "algorithmic 3 x 24405 FMA per increment (recomputed forward and "
                               "the two adjoint products); FP64 peak computed at 1965 MHz"}
    return res


def _backward_launch(mode, dt, n, L, w, d, inc, W, dev):
    """A closure running rpyb_signature_backward once on the given batch."""
    import torch
    from roughpy_b200 import _lib
    from roughpy_b200 import signatures as S
    off = np.arange(n + 1, dtype=np.int64) * L
    plan = S.SignaturePlan(off, w, d, mode, device=dev)
    x = torch.from_numpy(inc[:n * L]).to(dev, dt)
    G = W.to(dt).expand(n, plan.size).contiguous()
    ws = int(_lib.lib.rpyb_signature_backward_workspace_size(plan.code, w, d, n, L, 64))
    wsb = torch.empty(max(ws, 1), dtype=torch.uint8, device=dev)
    gi = torch.empty_like(x)

    def launch():
        _lib.check(_lib.lib.rpyb_signature_backward(
            plan.code, w, d, n, plan.offsets.data_ptr(), L, x.data_ptr(), G.data_ptr(),
            G.stride(0), gi.data_ptr(), 64, wsb.data_ptr(), ws,
            torch.cuda.current_stream(dev).cuda_stream))
        return gi
    return launch


def profile_backward(n):
    """One f32c adjoint launch on the first n streams of the 512 x 1024,
    width 5, depth 6 backward workload (the case captured by ncu)."""
    import torch
    L, w, d = 1024, 5, 6
    rng = np.random.default_rng(4)
    inc = rng.normal(0, np.sqrt(1.0 / L), size=(512 * L, w))
    T = (w ** (d + 1) - 1) // (w - 1)
    W = torch.from_numpy(rng.normal(size=(T,))).cuda()
    _backward_launch("f32c", torch.float32, n, L, w, d, inc, W, torch.device("cuda"))()
    torch.cuda.synchronize()
    print("profile backward done", n)


def profile_slice(n):
    """One f32c and one f64 signature launch on an n-stream slice of the bench
    workload (the case captured by ncu)."""
    import torch
    from roughpy_b200 import signatures as S
    lens, off, inc = make_workload(2, n)
    x32 = torch.from_numpy(inc).cuda()
    for mode, x in (("f32c", x32), ("f64", x32.double())):
        plan = S.SignaturePlan(off, WIDTH, DEPTH, mode)
        out = torch.empty((n, plan.size), dtype=plan.dtype, device="cuda")
        plan.run(x, out)
        torch.cuda.synchronize()
    print("profile slice done", n)


def profile_queries(nq, log2_events=16):
    """The dyadic-query workload's tree (2^16 events, width 6, depth 5,
    resolution 16, float32 nodes; 2^log2_events events at resolution
    log2_events for a smaller capture) and one query call of nq
    log-signatures: one fused chain-product, log and Hall-projection launch
    per chunk of 8192 queries (after the range-product table's launches when
    nq >= 1024)."""
    import torch
    from roughpy_b200.streams import LieIncrementStream
    n = 1 << log2_events
    rng = np.random.default_rng(3)
    inc = rng.normal(0, np.sqrt(1.0 / n), size=(n, 6)).astype(np.float32)
    idx = np.arange(n) / n
    q = np.sort(np.floor(rng.uniform(0, 1, size=(nq, 2)) * n) / n, axis=1)
    st = LieIncrementStream.from_increments(inc, indices=idx, width=6, depth=5,
                                            resolution=log2_events)
    st._build_tree()
    st.log_signature_batch(q[:, 0], q[:, 1])
    torch.cuda.synchronize()
    print("profile queries done", nq, log2_events)


def profile_fma(w, d, batch):
    """One float64 and one float32 C += A (x) B launch over `batch` pairs."""
    import torch
    from roughpy_b200 import _lib
    T = int(_lib.lib.rpyb_tensor_size(w, d))
    for dt, code in ((torch.float64, _lib.F64), (torch.float32, _lib.F32)):
        g = torch.Generator(device="cuda").manual_seed(1)
        A = torch.randn(batch, T, dtype=dt, device="cuda", generator=g)
        B = torch.randn(batch, T, dtype=dt, device="cuda", generator=g)
        C = torch.randn(batch, T, dtype=dt, device="cuda", generator=g)
        _lib.check(_lib.lib.rpyb_ft_fma(code, w, d, batch, C.data_ptr(), A.data_ptr(),
                                        B.data_ptr(), T, T, T, None, 0))
        torch.cuda.synchronize()
    print("profile fma done", w, d, batch)


# ------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    """Reference CPU implementation of the path (rank 0 only)."""
    if rank != 0:
        return None
    lens, off, inc = make_workload(seed=2)
    base = CpuBaseline()
    per_step = base.cores  # one stream per core per step
    rng = np.random.default_rng(123)
    order = rng.permutation(N_STREAMS)
    cursor = 0

    def next_sample():
        nonlocal cursor
        idx = order[cursor:cursor + per_step]
        cursor = (cursor + per_step) % (N_STREAMS - per_step)
        return sample_streams(inc, off, idx)

    for _ in range(args.warmup):
        base.run(next_sample())
    total, elapsed, steps_done = 0, 0.0, 0
    for _ in range(args.steps):
        n, dt = base.run(next_sample())
        total += n
        elapsed += dt
        steps_done += 1
    base.close()
    value = total / elapsed
    return {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "streams/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * elapsed / max(1, steps_done), 2),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Brownian increments)",
        "config": {
            "workload": "uneven batched signatures: lengths U{16..4096}, width 8, depth 5 "
                        "(bounded sample per step)",
            "width": WIDTH, "depth": DEPTH,
        },
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 3), "unit": "streams/s", "cores": base.cores,
                         "kind": base.kind,
                         "sample": f"{per_step} streams per step drawn from the 4096-stream "
                                   f"workload, chained roughpy.compute ft_fmexp in float64"},
        "e2e": {"value": round(value, 3), "unit": "streams/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def cpu_baseline_leg(workload):
    lens, off, inc = workload
    base = CpuBaseline()
    rng = np.random.default_rng(7)
    idx = rng.choice(len(lens), size=min(2 * base.cores, len(lens)), replace=False)
    n, dt = base.run(sample_streams(inc, off, idx))
    base.close()
    return {"value": round(n / dt, 3), "unit": "streams/s", "cores": base.cores,
            "kind": base.kind,
            "sample": f"{n} streams drawn at random from the 4096-stream workload "
                      f"(mean length {float(lens[idx].mean()):.0f}), chained ft_fmexp, "
                      f"float64, one process per core"}


def free_port() -> int:
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def relaunch_with_ranks(args) -> int:
    """`--gpus N` without a launcher: start N ranks on this node with
    torch.distributed.run (127.0.0.1 rendezvous) and return their status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1",
           f"--master-port={free_port()}", str(pathlib.Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="weak: 4096 streams per GPU; strong: one 4096-stream batch sharded")
    ap.add_argument("--dry-run", action="store_true",
                    help="exercise the rank plumbing on CPU (gloo) without computing")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the plain-f64, long-stream, dyadic-query and backward workloads")
    ap.add_argument("--profile-backward", type=int, default=0,
                    help="run one adjoint launch on N streams of the backward workload and exit")
    ap.add_argument("--profile-slice", type=int, default=0,
                    help="run one launch per mode on an N-stream slice and exit")
    ap.add_argument("--profile-fma", type=int, nargs=3, metavar=("WIDTH", "DEPTH", "BATCH"),
                    help="run one float64 and one float32 FMA launch and exit")
    ap.add_argument("--profile-queries", type=int, nargs="+", metavar=("N", "LOG2_EVENTS"),
                    help="build the dyadic-query tree (2^16 events unless given), run N "
                         "queries and exit")
    args = ap.parse_args()
    if args.profile_backward:
        profile_backward(args.profile_backward)
        return
    if args.profile_slice:
        profile_slice(args.profile_slice)
        return
    if args.profile_fma:
        profile_fma(*args.profile_fma)
        return
    if args.profile_queries:
        profile_queries(*args.profile_queries[:2])
        return
    if args.warmup < 3 and args.impl == "b200":
        log("note: warmup raised to 3")
        args.warmup = 3

    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(relaunch_with_ranks(args))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return

    import datetime
    import torch
    import torch.distributed as dist
    if args.dry_run:
        if world > 1:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        try:
            res = dry_run(args, rank, world)
            if res is not None:
                print(json.dumps(res), flush=True)
        finally:
            if world > 1:
                dist.barrier()
                dist.destroy_process_group()
        return
    if world > 1:
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        res, workload = run_b200(args, rank, world, local_rank)
        if rank == 0:
            if not args.no_extra:
                dev = torch.device("cuda", local_rank)
                for key, fn in (("plain_f64_signatures", plain_f64_signatures),
                                ("long_streams", long_streams),
                                ("dyadic_queries", dyadic_queries),
                                ("signature_backward", signature_backward)):
                    try:
                        res[key] = fn(dev)
                    except Exception as exc:  # keep the headline line
                        res[key] = {"error": f"{type(exc).__name__}: {exc}"}
            if not args.no_cpu:
                res["cpu_baseline"] = cpu_baseline_leg(workload)
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
