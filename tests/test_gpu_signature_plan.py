"""Signature plans (rpyb_sig_plan): schedules, time-segment splitting of long
streams, and the tuning cache.

* Segmented long streams (the Chen product of the segment signatures, in
  order) against the C oracle in float64 <= 1e-12, and the float32 path
  against float64 <= 1e-6.
* Lane shapes and block sizes change only how words are dealt to lanes, so
  every forced schedule without segments gives bitwise identical results.
* Tuning writes the chosen schedule to the cache file named by
  RPYB_SIG_TUNE_CACHE and a second plan of the same bucket reads it.
"""
import json
import os

import numpy as np
import pytest
import torch

import oracle
from roughpy_b200 import signatures as S
from tests._util import level_rel_err

pytestmark = pytest.mark.gpu


class forced:
    """Sets RPYB_SIG_SCHEDULE (read at plan creation) for a with-block."""

    def __init__(self, value):
        self.value = value

    def __enter__(self):
        self.old = os.environ.get("RPYB_SIG_SCHEDULE")
        os.environ["RPYB_SIG_SCHEDULE"] = self.value

    def __exit__(self, *exc):
        if self.old is None:
            del os.environ["RPYB_SIG_SCHEDULE"]
        else:
            os.environ["RPYB_SIG_SCHEDULE"] = self.old


def test_segmented_long_streams_float64_against_oracle():
    """8 streams of 2^17 increments at width 4, depth 5, cut into 4096-step
    segments (32 per stream, five merge levels)."""
    rng = np.random.default_rng(41)
    w, d, n, L = 4, 5, 8, 1 << 17
    off = np.arange(n + 1, dtype=np.int64) * L
    inc = rng.normal(0, np.sqrt(1.0 / L), size=(n * L, w))
    with forced("seg=4096"):
        plan = S.SignaturePlan(off, w, d, "f64")
    sch = plan.schedule()
    assert sch["seg"] == 4096 and sch["items"] == n * 32 and sch["merge_levels"] == 5
    got = plan.run(torch.from_numpy(inc).cuda()).cpu().numpy()
    for s in range(n):
        want = oracle.signature(w, d, inc[off[s]:off[s + 1]])
        assert level_rel_err(got[s], want, w, d) <= 1e-12, s


@pytest.mark.parametrize("seg", [1000, 4096])
def test_segmented_uneven_float32_against_unsplit_float64(seg):
    """Width 8, depth 5, a mix of short and long streams (some split into an
    odd number of segments, some not split)."""
    rng = np.random.default_rng(seg)
    w, d = 8, 5
    lens = np.array([50000, 3, 0, 9000, 12001, 700, 4096, 4097, 20000])
    off = S.offsets_from_lengths(lens)
    inc = np.concatenate([rng.normal(0, np.sqrt(1.0 / max(L, 1)), size=(L, w)) for L in lens])
    x32 = torch.from_numpy(inc.astype(np.float32)).cuda()
    with forced(f"seg={seg}"):
        plan = S.SignaturePlan(off, w, d, "f32c")
        plan64 = S.SignaturePlan(off, w, d, "f64")
    assert plan.schedule()["seg"] == seg
    got, err = plan.run(x32, report_error=True)
    with forced("seg=0"):
        ref = S.SignaturePlan(off, w, d, "f64").run(x32.double())
    seg64 = plan64.run(x32.double())
    torch.cuda.synchronize()
    g, r = got.cpu().numpy(), ref.cpu().numpy()
    assert level_rel_err(g, r, w, d) <= 1e-6
    assert float(err.max()) <= 1e-6
    # the segmented float64 result is the same product, reassociated
    assert level_rel_err(seg64.cpu().numpy(), r, w, d) <= 1e-12
    # empty stream: unit tensor
    assert g[2, 0] == 1.0 and not np.any(g[2, 1:])


@pytest.mark.parametrize("mode,w,d,scheds", [
    ("f32c", 8, 5, ["g=8,wpb=0", "g=4,wpb=0", "g=8,wpb=4", "g=4,wpb=2"]),
    ("f64", 8, 5, ["g=8", "g=4,wpb=4"]),
    ("f32c", 6, 5, ["g=6", "g=3,wpb=4"]),
    ("f32c", 4, 6, ["g=4", "g=2,wpb=1"]),
    ("f64", 4, 6, ["g=4", "g=2"]),
])
def test_lane_shapes_and_block_sizes_are_bitwise_identical(mode, w, d, scheds):
    rng = np.random.default_rng(w * d)
    lens = rng.integers(0, 600, size=33)
    off = S.offsets_from_lengths(lens)
    dt = torch.float64 if mode == "f64" else torch.float32
    x = torch.from_numpy(rng.normal(0, 0.05, size=(int(off[-1]), w))).to("cuda", dt)
    outs = []
    for sc in scheds:
        with forced(sc + ",seg=0"):
            plan = S.SignaturePlan(off, w, d, mode)
        g = int(sc.split(",")[0].split("=")[1])
        assert plan.schedule()["g"] == g
        outs.append(plan.run(x))
    torch.cuda.synchronize()
    for o in outs[1:]:
        assert torch.equal(o, outs[0])


def test_tuning_writes_and_reads_the_cache(tmp_path, monkeypatch):
    cache = tmp_path / "schedules.json"
    monkeypatch.setenv("RPYB_SIG_TUNE_CACHE", str(cache))
    monkeypatch.delenv("RPYB_SIG_SCHEDULE", raising=False)
    rng = np.random.default_rng(3)
    w, d = 8, 4
    lens = rng.integers(1000, 3000, size=4)
    off = S.offsets_from_lengths(lens)
    plan = S.SignaturePlan(off, w, d, "f32c", tune=True)
    first = plan.schedule()
    assert first["source"] == "tuned" and first["ms"] > 0
    data = json.loads(cache.read_text())
    assert first["key"] in data
    assert data[first["key"]]["g"] == first["g"]
    again = S.SignaturePlan(off, w, d, "f32c", tune=True).schedule()
    assert again["source"] == "cache"
    assert (again["g"], again["wpb"], again["seg"]) == (first["g"], first["wpb"], first["seg"])
    x = torch.from_numpy(rng.normal(0, 0.03, size=(int(off[-1]), w)).astype(np.float32)).cuda()
    got = plan.run(x)
    ref = S.SignaturePlan(off, w, d, "f64", tune=False).run(x.double())
    torch.cuda.synchronize()
    assert level_rel_err(got.cpu().numpy(), ref.cpu().numpy(), w, d) <= 1e-6
