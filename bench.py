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
SM_COUNT_B200 = 148
FP32_LANES_PER_SM = 128
# dram bytes per launch of the float32 signature kernel on this workload,
# from the ncu capture summarised in profiles/signature_f32c_w8d5.md
# (captured on a 512-stream slice; DRAM traffic scales with the stream count).
SIG_TRAFFIC_BYTES_PER_STREAM = None


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


# ------------------------------------------------------------- GPU arm
def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from roughpy_b200 import signatures as S
    from roughpy_b200 import _lib

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lens, off, inc = make_workload(seed=2 + rank)
    T = S.tensor_size(WIDTH, DEPTH)
    inc_d = torch.from_numpy(inc).to(dev)
    plan = S.SignaturePlan(off, WIDTH, DEPTH, "f32c", device=dev)
    out_d = torch.empty((N_STREAMS, T), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

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
    clk = clocks.stop() if clocks else None
    ms_total = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = ms_total / args.steps
    value = world * N_STREAMS / (ms_step / 1e3)

    # ---- end to end through the C ABI from pinned host buffers
    inc_h = torch.from_numpy(inc).pin_memory()
    out_h = torch.empty((N_STREAMS, T), dtype=torch.float32).pin_memory()
    for _ in range(args.warmup):
        plan.run_host(inc_h, out_h, inc_d, out_d)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.run_host(inc_h, out_h, inc_d, out_d)
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    e2e_value = world * N_STREAMS / (e2e_ms / 1e3)

    # ---- float64 path on the same inputs: speed and the accuracy of float32
    plan64 = S.SignaturePlan(off, WIDTH, DEPTH, "f64", device=dev)
    inc64 = inc_d.double()
    out64 = torch.empty((N_STREAMS, T), dtype=torch.float64, device=dev)
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
    plan.run(inc_d, out_d)
    torch.cuda.synchronize(dev)
    err = max_over_ranks(level_rel_err_torch(out_d, out64, WIDTH, DEPTH))

    result = None
    if rank == 0:
        pk, pk_kind = peaks()
        sm_mhz = (clk or {}).get("sm_mhz") or pk.get("sm_max_mhz", 1965.0)
        fp32_peak = 2 * FP32_LANES_PER_SM * SM_COUNT_B200 * sm_mhz * 1e6 / 1e12
        algo_flops = 2.0 * FMA_PER_STEP * float(lens.sum())
        achieved = algo_flops / (ms_step / 1e3) / 1e12 / world * world  # per GPU
        achieved = algo_flops / (ms_step / 1e3) / 1e12
        traffic = (SIG_TRAFFIC_BYTES_PER_STREAM * N_STREAMS
                   if SIG_TRAFFIC_BYTES_PER_STREAM else None)
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
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (compensated)",
            "data": "synthetic (seeded Brownian increments)",
            "config": {
                "workload": "uneven batched signatures: 4096 streams/GPU, lengths U{16..4096}, "
                            "width 8, depth 5, increments N(0,1/len), FP32-comp",
                "global_batch": world * N_STREAMS,
                "width": WIDTH, "depth": DEPTH,
                "parallelism": f"dp{world} (streams sharded, no collective)",
                "l2": "inputs+outputs 0.9 GB per step > 126 MB L2 (no flush needed)",
            },
            "f64_path": {"value": round(world * N_STREAMS / (ms64 / 1e3), 1),
                         "unit": "streams/s", "ms_per_step": round(ms64, 4)},
            "f32c_speedup_vs_f64": round(ms64 / ms_step, 3),
            "max_rel_err_vs_f64": err,
            "roofline": {
                "bound": "fp32_fma", "achieved": round(achieved, 3), "peak": round(fp32_peak, 2),
                "unit": "TFLOP/s", "frac": round(achieved / fp32_peak, 4),
                "traffic": traffic,
                "note": "algorithmic 2*42792 flop per increment; FP32 CUDA-core peak "
                        "= 148 SM x 128 lanes x 2 x sampled SM clock (no tensor cores on "
                        "this path)",
            },
            "tensor_mul": sweep,
            "e2e": {"value": round(e2e_value, 1), "unit": "streams/s",
                    "h2d_bytes_per_step": int(inc.nbytes),
                    "d2h_bytes_per_step": int(N_STREAMS * T * 4),
                    "ms_per_step": round(e2e_ms, 4)},
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
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = 10
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / reps
            gbs = 4.0 * T * es * SWEEP_BATCH / (ms / 1e3) / 1e9
            res[f"w{w}d{d}_{name}"] = {"ms": round(ms, 4), "GB/s": round(gbs, 1),
                                       "frac_hbm": round(gbs / hbm_gbs, 3)}
            del A, B, C
    torch.cuda.empty_cache()
    return res


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
    idx = rng.choice(N_STREAMS, size=2 * base.cores, replace=False)
    n, dt = base.run(sample_streams(inc, off, idx))
    base.close()
    return {"value": round(n / dt, 3), "unit": "streams/s", "cores": base.cores,
            "kind": base.kind,
            "sample": f"{n} streams drawn at random from the 4096-stream workload "
                      f"(mean length {float(lens[idx].mean()):.0f}), chained ft_fmexp, "
                      f"float64, one process per core"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        log("note: warmup raised to 3")
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        res, workload = run_b200(args, rank, world, local_rank)
        if rank == 0:
            if not args.no_cpu:
                res["cpu_baseline"] = cpu_baseline_leg(workload)
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
