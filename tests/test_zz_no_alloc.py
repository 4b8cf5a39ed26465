"""dg_read_cells_noalloc, the allocation-free cell read-back, against dg_read_cells.

Hosts that own all device memory through their own allocator, or threads that must not take the
device-wide synchronisation of cudaMalloc, read the solver state through this entry point; it
gathers through a fixed 64 MiB scratch array kept by the library instead of allocating. This file
runs last so that a failure here leaves the rest of the suite already run.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from dacti_b200 import cases
from dacti_b200.casefile import read_case
from dacti_b200.solver import DgError, Solver

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _same(a, b):
    assert a.n == b.n
    assert np.array_equal(a.tree_level, b.tree_level) and np.array_equal(a.acti_level, b.acti_level)
    for x, y in ((a.u, b.u), (a.p, b.p), (a.center, b.center), (a.t, b.t)):
        assert np.all(np.abs(x - y) <= TOL * np.maximum(np.abs(x), 1.0))


def test_noalloc_read_matches_allocating_read_twice():
    case = read_case(os.path.join(GOLDEN, "multi2.case"))
    s = Solver(case)
    for _ in range(2):
        s.integrate()
        _same(s.active_cells(), s.active_cells_noalloc())
    s.close()


def test_noalloc_first_call_on_a_fresh_solver_allocates_nothing():
    """The scratch array and the gather kernel are placed on the device by dg_create, so the first
    read-back of a new solver leaves the device's free memory where it was."""
    import torch

    case = cases.shock_drop(base_level=3, levels=2)
    s = Solver(case)
    s.integrate()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    snap = s.active_cells_noalloc()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert snap.n == s.n_active_cells() > 0
    _same(s.active_cells(), snap)
    s.close()


def test_noalloc_read_rejects_more_cells_than_its_scratch_holds():
    case = cases.lax_liu3(base_level=10, levels=0)  # 2^20 euler<2> cells
    s = Solver(case)
    with pytest.raises(DgError) as e:
        s.active_cells_noalloc()
    # euler<2>: 8 (D + 2E + P + 5) = 120 bytes per cell of the 64 MiB scratch (256 bytes of alignment slack)
    assert e.value.code == -3 and "scratch" in str(e.value)
    assert f"about {((64 << 20) - 256) // 120} cells" in str(e.value)
    assert s.active_cells().n == 1 << 20
    s.close()
