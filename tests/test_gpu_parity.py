"""GPU parity with the reference solver: identical refinement decisions and ACTI levels, conserved
fields within rel-L1 1e-10 (FP64 plain form)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, run_reference
from dacti_b200 import cases
from dacti_b200.casefile import read_case, read_snapshot, write_case
from dacti_b200.parity import compare
from dacti_b200.solver import Solver
from tests.golden.make_golden import GOLDEN as CASES

pytestmark = pytest.mark.gpu
TOL = 1e-10  # relative L1 of every conserved component


def _run(case, steps, checks):
    s = Solver(case)
    out = {}
    if 0 in checks:
        out[0] = s.active_cells()
    for k in range(1, steps + 1):
        _, fb = s.integrate()
        assert not fb
        if k in checks:
            out[k] = s.active_cells()
    stats = s.stats()
    s.close()
    return out, stats


def _keyed(snap, side):
    return snap.sorted(side)


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if 0 in CASES[n][2]])
def test_construction_is_bit_exact(name):
    """After the Integrator constructor (integrator/integrator.hpp:100-160) every cell's conserved
    state, slopes' products and the multiphase parameters (smoothed volume fraction, interface normal,
    curvature) equal the reference bit for bit: same inputs, same operation order, no accumulation."""
    _, steps, checks = CASES[name]
    case = read_case(os.path.join(GOLDEN, f"{name}.case"))
    got, _ = _run(case, 0, [0])
    ref = read_snapshot(os.path.join(GOLDEN, f"{name}_0.snap"))
    side = case.params.side_length
    a, b = ref.sorted(side), got[0].sorted(side)
    assert a.n == b.n
    assert np.array_equal(a.u, b.u) and np.array_equal(a.p, b.p)
    assert np.array_equal(a.acti_level, b.acti_level) and np.array_equal(a.max_dt, b.max_dt)
    if a.k is not None:
        D = case.shape.dims
        kappa = 2 + D
        # interface normals and smoothed volume fraction
        assert np.array_equal(a.k[:, 2:2 + D], b.k[:, 2:2 + D]) and np.array_equal(a.k[:, kappa + 1], b.k[:, kappa + 1])
        # the curvature only matters, and is only computed, with surface tension
        if case.params.sigma != 0.0:
            assert np.array_equal(a.k[:, kappa], b.k[:, kappa])


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if CASES[n][1] > 0])
def test_golden_parity(name):
    _, steps, checks = CASES[name]
    case = read_case(os.path.join(GOLDEN, f"{name}.case"))
    got, _ = _run(case, steps, checks)
    for k in checks:
        ref = read_snapshot(os.path.join(GOLDEN, f"{name}_{k}.snap"))
        rep = compare(ref, got[k], case.params.side_length)
        assert rep.ok(TOL), f"{name} step {k}: {rep}"
        assert got[k].n == ref.n


def _live(case, steps, checks, tmp_path, name, threads=1):
    path = str(tmp_path / f"{name}.case")
    write_case(case, path)
    run_reference(path, str(tmp_path / name), steps, checks, threads=threads)
    got, stats = _run(case, steps, checks)
    for k in checks:
        ref = read_snapshot(str(tmp_path / f"{name}_{k}.snap"))
        rep = compare(ref, got[k], case.params.side_length)
        assert rep.ok(TOL), f"{name} step {k}: {rep}"
        assert stats.cell_updates >= ref.updates or k != checks[-1]
    return stats


def test_lax_liu_config1_full_run(tmp_path):
    """Config 1 at its full size (64^2 base, +3 levels) for the 26 global steps to t = 0.309."""
    stats = _live(cases.lax_liu3(), 26, [1, 13, 26], tmp_path, "c1")
    assert stats.n_global_steps == 26


def test_garbage_collection_run(tmp_path):
    """A run long enough for the reference's memory-efficiency trigger to compact the tree."""
    stats = _live(cases.lax_liu3(base_level=5, levels=3), 43, [20, 43], tmp_path, "gc")
    assert stats.n_gc >= 1


def test_multi3_larger(tmp_path):
    _live(cases.shock_drop(base_level=4, levels=2), 3, [1, 3], tmp_path, "sd3")


def test_shock_drop_config2_reduced(tmp_path):
    """Config 2's shock-drop at a quarter of its base resolution per axis (32 x 16 x 16 base, +3 levels,
    a 6.4e5-node initial tree) for 2 global steps against the single-thread reference."""
    stats = _live(cases.shock_drop(base_level=5, levels=3), 2, [1, 2], tmp_path, "sd53")
    assert stats.n_substeps > 100


def test_cylinder_config4_stated_size(tmp_path):
    """Config 4's Navier-Stokes cylinder at its stated size (128 x 64 base, the power-of-two grid nearest
    80 x 40, +5 levels; no-slip solid, Re 200) for 6 global steps against the single-thread reference."""
    stats = _live(cases.cylinder_ns(mach=0.3, base_level=7, levels=5), 6, [3, 6], tmp_path, "cyl75")
    assert stats.n_substeps > 500


def test_periodic_without_refinement(tmp_path):
    _live(cases.periodic_blob(base_level=5, refine=False), 8, [8], tmp_path, "pnr")


@pytest.mark.parametrize("which", ["shock_drop", "cylinder"])
def test_pruned_upload_gives_the_same_results(which):
    """A tree uploaded without its inactive subtrees (casefile.prune_inactive) steps to the same cells,
    ACTI levels and conserved state bit for bit, with the same tree size and garbage collections."""
    from dacti_b200.casefile import prune_inactive
    case = (cases.shock_drop(base_level=4, levels=2) if which == "shock_drop"
            else cases.cylinder_ns(mach=0.3, base_level=4, levels=2))
    steps = 4 if which == "shock_drop" else 12
    out = []
    for c in (case, prune_inactive(case)):
        s = Solver(c)
        for _ in range(steps):
            assert not s.integrate()[1]
        out.append((s.active_cells().sorted(case.params.side_length), s.stats()))
        s.close()
    (a, sa), (b, sb) = out
    assert a.n == b.n and np.array_equal(a.u, b.u) and np.array_equal(a.acti_level, b.acti_level)
    assert sa.tree_size == sb.tree_size and sa.n_gc == sb.n_gc and sa.cell_updates == sb.cell_updates


def test_bitwise_determinism():
    case = read_case(os.path.join(GOLDEN, "multi2.case"))
    a, _ = _run(case, 4, [4])
    b, _ = _run(case, 4, [4])
    sa, sb = a[4].sorted(case.params.side_length), b[4].sorted(case.params.side_length)
    assert np.array_equal(sa.u, sb.u) and np.array_equal(sa.p, sb.p)


def test_nan_state_sets_force_break():
    """Fault injection on the host: one cell with negative density makes the step report NaN."""
    case = cases.lax_liu3(base_level=4, levels=1)
    leaves = np.nonzero(case.tree.leaf_mask())[0]
    case.tree.p[leaves[37], 0] = -1.0
    s = Solver(case)
    _, fb = s.integrate()
    s.close()
    assert fb
