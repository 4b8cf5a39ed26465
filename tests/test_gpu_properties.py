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


@pytest.mark.parametrize("name,steps,level", [("multi2", 4, 4), ("multi3", 2, 3), ("euler2", 6, 3), ("ns2", 6, 3)])
def test_mixed_form_density_error_vs_fp64(name, steps, level):
    """FP32 reconstruction and flux with FP64 update: mixture-density rel-L1 against the FP64 form on
    the uniform base grid stays within 1e-4."""
    import os

    from conftest import GOLDEN
    from dacti_b200.accuracy import density_rel_l1
    from dacti_b200.casefile import read_case

    case = read_case(os.path.join(GOLDEN, f"{name}.case"))
    snaps = {}
    for form in ("fp64", "mixed"):
        s = Solver(case)
        s.set_form(form)
        for _ in range(steps):
            _, fb = s.integrate()
            assert not fb
        snaps[form] = s.active_cells()
        s.close()
    err = density_rel_l1(snaps["mixed"], snaps["fp64"], case.params.side_length, case.params.active_size, level,
                         int(case.shape.model))
    assert err <= 1e-4, err
    assert err > 0.0


def test_mixed_form_conservation_without_refinement():
    """Both cells of a face evaluate the same FP32 flux, so the FP64 totals stay conserved."""
    case = cases.periodic_blob(base_level=6, refine=False)
    s = Solver(case)
    s.set_form("mixed")
    t0 = _totals(s.active_cells(), 1.0, 2)
    for _ in range(5):
        s.integrate()
    t1 = _totals(s.active_cells(), 1.0, 2)
    s.close()
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0))
