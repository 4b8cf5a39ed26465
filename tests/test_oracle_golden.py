"""The reference oracle (DACTI's own Integrator built from its sources) reproduces its golden fixtures.

The fixtures under tests/golden were written by tests/golden/make_golden.py with the same runner;
re-running it here pins the oracle build bit for bit (single thread, no FMA contraction), so a
parity claim against the oracle is a claim against these committed outputs.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, run_reference
from dacti_b200.casefile import read_snapshot
from tests.golden.make_golden import GOLDEN as CASES


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_golden(name, tmp_path):
    _, steps, checks = CASES[name]
    run_reference(os.path.join(GOLDEN, f"{name}.case"), str(tmp_path / name), max(steps, 0), checks)
    for k in checks:
        got = read_snapshot(str(tmp_path / f"{name}_{k}.snap"))
        ref = read_snapshot(os.path.join(GOLDEN, f"{name}_{k}.snap"))
        assert got.n == ref.n
        assert np.array_equal(got.tree_level, ref.tree_level)
        assert np.array_equal(got.acti_level, ref.acti_level)
        assert np.array_equal(got.u, ref.u)
        assert np.array_equal(got.p, ref.p)
        assert got.updates == ref.updates
