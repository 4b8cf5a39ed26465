import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
RUNNER = os.path.join(ROOT, "oracle", "_ref", "dacti_ref_runner")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def run_reference(case_path: str, out_prefix: str, steps: int, checks, threads: int = 1, extra=()) -> str:
    """Runs the reference solver built from its own sources; returns its JSON summary line."""
    if not os.path.exists(RUNNER):
        pytest.fail(f"reference runner missing: {RUNNER} (build with `make -C oracle`)")
    r = subprocess.run([RUNNER, case_path, out_prefix, str(steps), "--check", ",".join(map(str, checks)), *extra],
                       capture_output=True, text=True, env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout.strip()
