"""bench.py's multi-rank plumbing on CPU: `--gpus 2` with no launcher starts two
ranks through torch.distributed.run (gloo in --dry-run), every rank builds its
workload and shard, the timing is the max over ranks, and rank 0 alone prints
one JSON line with n_gpus = 2.  The dry run computes nothing (its step copies
the rank's rows on the host)."""
import json
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def run_bench(*extra):
    cmd = [sys.executable, str(ROOT / "bench.py"), "--dry-run", "--gpus", "2", "--steps", "2",
           "--warmup", "3", *extra]
    proc = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [ln for ln in proc.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, proc.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("scaling", ["strong", "weak"])
def test_two_ranks_report_one_line(scaling):
    res = run_bench("--scaling", scaling)
    assert res["n_gpus"] == 2 and res["dry_run"] is True
    assert res["scaling"] == scaling
    shards = res["config"]["shards"]
    assert len(shards) == 2
    if scaling == "strong":
        # contiguous, length-balanced shards tiling the one 4096-stream batch
        assert shards[0][0] == 0 and shards[0][1] == shards[1][0] and shards[1][1] == 4096
        assert res["config"]["global_batch"] == 4096
    else:
        assert shards == [[0, 4096], [0, 4096]]
        assert res["config"]["global_batch"] == 8192
    assert res["value"] > 0 and res["ms_per_step"] > 0
