"""The reference's own `tests/compute` files, unmodified, against the drop-in
`roughpy_b200.compute` (aliased as `roughpy.compute` by
tests/reference_alias.py).  The files are not part of this repository: point
RPYB_REFERENCE_TESTS at a directory holding them (the reference checkout's
tests/compute); the test is skipped otherwise.  The shuffle tests need the
reference's main-library fixtures (its top-level conftest imports the
unbuildable `roughpy._roughpy`) and are left out."""
import os
import pathlib
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parent.parent


def test_reference_compute_suite_passes_against_the_drop_in():
    src = os.environ.get("RPYB_REFERENCE_TESTS")
    if not src:
        pytest.skip("RPYB_REFERENCE_TESTS is not set")
    files = sorted(str(p) for p in pathlib.Path(src).glob("test_*.py")
                   if p.name != "test_shuffle.py")
    assert files, f"no test files under {src}"
    env = dict(os.environ, PYTHONPATH=str(ROOT) + os.pathsep + os.environ.get("PYTHONPATH", ""))
    cmd = [sys.executable, "-m", "pytest", "-q", "-p", "tests.reference_alias", "--noconftest",
           "-o", "addopts=", "--rootdir", src, "-p", "no:cacheprovider", *files]
    proc = subprocess.run(cmd, capture_output=True, text=True, env=env, cwd=str(ROOT), timeout=1200)
    print(proc.stdout[-3000:])
    assert proc.returncode == 0, proc.stdout[-3000:] + proc.stderr[-2000:]
    assert " passed" in proc.stdout and " failed" not in proc.stdout
