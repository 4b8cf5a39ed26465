"""Size-independent properties at the benchmark's full size and conservation without refinement."""
import numpy as np
import pytest

from dacti_b200 import cases
from dacti_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _totals(snap, side, D):
    vol = (side * 0.5 ** snap.tree_level.astype(np.float64)) ** D
    return (snap.u * vol[:, None]).sum(axis=0)


def test_periodic_conservation_without_refinement():
    """Mass, momentum and energy of a closed periodic box are conserved by the flux/update stages."""
    case = cases.periodic_blob(base_level=6, refine=False)
    s = Solver(case)
    t0 = _totals(s.active_cells(), 1.0, 2)
    for _ in range(5):
        s.integrate()
    t1 = _totals(s.active_cells(), 1.0, 2)
    s.close()
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0))


def test_shock_drop_full_size_step():
    """Config 2 at full size (64 x 32 x 32 base, +4 levels): one global step stays finite and ends with
    every cell at the same time."""
    case = cases.shock_drop()
    s = Solver(case)
    gdt, fb = s.integrate()
    snap = s.active_cells()
    st = s.stats()
    s.close()
    assert not fb
    assert np.isfinite(snap.u).all() and np.isfinite(snap.p).all()
    assert snap.n > 1_000_000
    assert np.max(np.abs(snap.t - gdt)) <= 1e-12 * gdt
    assert st.cell_updates > 10 * snap.n
    a = snap.p[:, case.shape.ia]
    assert a.min() >= -1e-12 and a.max() <= 1 + 1e-12
