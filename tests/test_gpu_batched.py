"""Batched trees (dg_step_many and the lockstep dg_batch): independent quadtree Riemann problems stepped
concurrently give, tree by tree, exactly the results of stepping each tree alone, and those match the
reference solver run on each tree (one Integrator per tree)."""
import numpy as np
import pytest

from conftest import run_reference
from dacti_b200 import cases
from dacti_b200.casefile import read_snapshot, write_case
from dacti_b200.parity import compare
from dacti_b200.solver import Batch, Solver, step_many

pytestmark = pytest.mark.gpu
STEPS = 3


def _batch():
    return cases.riemann_batch(12, seed=11, base_levels=(4, 5), extra_levels=(2, 2))


def test_batched_steps_equal_single_tree_steps():
    batch = _batch()
    together = [Solver(c) for c in batch]
    alone = [Solver(c) for c in batch]
    for _ in range(STEPS):
        fb_t = step_many(together, threads=8)
        fb_a = [s.integrate()[1] for s in alone]
        assert fb_t == fb_a
    for a, b, c in zip(together, alone, batch):
        # list order depends on scheduling; the per-cell results do not
        sa, sb = a.active_cells().sorted(c.params.side_length), b.active_cells().sorted(c.params.side_length)
        assert sa.n == sb.n
        assert np.array_equal(sa.u, sb.u, equal_nan=True) and np.array_equal(sa.acti_level, sb.acti_level)
        assert a.stats().cell_updates == b.stats().cell_updates
    for s in together + alone:
        s.close()


@pytest.mark.parametrize("tree", [0, 3, 4, 11])
def test_batched_trees_match_reference(tree, tmp_path):
    batch = _batch()
    solvers = [Solver(c) for c in batch]
    for _ in range(STEPS):
        step_many(solvers, threads=8)
    path = str(tmp_path / "t.case")
    write_case(batch[tree], path)
    run_reference(path, str(tmp_path / "t"), STEPS, [STEPS])
    ref = read_snapshot(str(tmp_path / f"t_{STEPS}.snap"))
    rep = compare(ref, solvers[tree].active_cells(), batch[tree].params.side_length)
    assert rep.ok(1e-10), rep
    for s in solvers:
        s.close()


def test_batch_extreme_trees_match_reference(tmp_path):
    """The largest (256^2 base, +4 levels) and the smallest (32^2 base, +2 levels) trees of the
    256-tree batch of the batched workload (cases.riemann_batch(256, seed=3)), stepped together with
    the lockstep batch (dg_batch) for 2 global steps, against the reference solver on each tree."""
    from dacti_b200.batch import tree_work
    full = cases.riemann_batch(256, seed=3)
    work = [tree_work(c) for c in full]
    pick = [int(np.argmax(work)), int(np.argmin(work))]
    assert full[pick[0]].params.min_level == 8 and full[pick[0]].params.max_level == 12
    steps = 2
    solvers = [Solver(full[k]) for k in pick]
    b = Batch(solvers)
    for _ in range(steps):
        assert not any(b.step())
    b.close()
    for s, k in zip(solvers, pick):
        path = str(tmp_path / f"t{k}.case")
        write_case(full[k], path)
        run_reference(path, str(tmp_path / f"t{k}"), steps, [steps])
        ref = read_snapshot(str(tmp_path / f"t{k}_{steps}.snap"))
        rep = compare(ref, s.active_cells(), full[k].params.side_length)
        assert rep.ok(1e-10), f"tree {k}: {rep}"
        s.close()


def test_lockstep_batch_equals_single_tree_steps():
    """dg_batch (merged schedules, one launch per stage for all trees) gives every tree's dg_step result
    bit for bit: cells, ACTI levels, conserved state, counters."""
    batch = cases.riemann_batch(12, seed=11, base_levels=(4, 6), extra_levels=(2, 3))
    together = [Solver(c) for c in batch]
    alone = [Solver(c) for c in batch]
    b = Batch(together)
    for _ in range(STEPS):
        fb_t = b.step()
        fb_a = [s.integrate()[1] for s in alone]
        assert fb_t == fb_a
    b.close()
    for a, s, c in zip(together, alone, batch):
        sa, sb = a.active_cells().sorted(c.params.side_length), s.active_cells().sorted(c.params.side_length)
        assert sa.n == sb.n
        assert np.array_equal(sa.u, sb.u, equal_nan=True) and np.array_equal(sa.acti_level, sb.acti_level)
        ta, tb = a.stats(), s.stats()
        assert ta.cell_updates == tb.cell_updates and ta.n_substeps == tb.n_substeps
        assert ta.n_splits == tb.n_splits and ta.n_unsplits == tb.n_unsplits
        assert ta.tree_size == tb.tree_size and ta.global_dt == tb.global_dt
    for s in together + alone:
        s.close()


def test_lockstep_batch_stops_and_resumes():
    """Pools with no room to spare: the planned runs stop at the capacity check, the host grows the pool,
    completes the substep and resumes, and every tree still gets its dg_step result bit for bit."""
    import dataclasses
    batch = [dataclasses.replace(c, params=dataclasses.replace(c.params, pool_capacity=1))
             for c in cases.riemann_batch(6, seed=5, base_levels=(4, 5), extra_levels=(2, 3))]
    together = [Solver(c) for c in batch]
    alone = [Solver(c) for c in batch]
    b = Batch(together)
    b.set_pregrow(False)
    for _ in range(STEPS):
        assert b.step() == [s.integrate()[1] for s in alone]
    st = b.run_stats()
    b.close()
    assert st["stops"] > 0 and st["completed"] > 0 and st["runs"] >= STEPS
    for a, s, c in zip(together, alone, batch):
        sa, sb = a.active_cells().sorted(c.params.side_length), s.active_cells().sorted(c.params.side_length)
        assert sa.n == sb.n
        assert np.array_equal(sa.u, sb.u, equal_nan=True) and np.array_equal(sa.acti_level, sb.acti_level)
        ta, tb = a.stats(), s.stats()
        assert (ta.cell_updates, ta.n_substeps, ta.n_splits, ta.n_unsplits, ta.tree_size) == \
            (tb.cell_updates, tb.n_substeps, tb.n_splits, tb.n_unsplits, tb.tree_size)
    for s in together + alone:
        s.close()


def test_lockstep_batch_force_breaks_equal_single_tree_steps():
    """Config 3's quadrant states drive some trees to a NaN pressure (force_break). A NaN tree halts on the
    device for the rest of the global step while the other trees run on; every tree, the halted ones
    included, still gets its dg_step result bit for bit, force_break flags and global dt too."""
    batch = cases.riemann_batch(24, seed=3, base_levels=(4, 5), extra_levels=(2, 3))
    together = [Solver(c) for c in batch]
    alone = [Solver(c) for c in batch]
    b = Batch(together)
    breaks = 0
    for _ in range(STEPS):
        fb_t = b.step()
        fb_a = [s.integrate()[1] for s in alone]
        assert fb_t == fb_a
        breaks += sum(fb_t)
        assert [s.global_dt for s in together] == [s.global_dt for s in alone]
    b.close()
    assert breaks > 0
    for a, s, c in zip(together, alone, batch):
        sa, sb = a.active_cells().sorted(c.params.side_length), s.active_cells().sorted(c.params.side_length)
        assert sa.n == sb.n
        assert np.array_equal(sa.u, sb.u, equal_nan=True) and np.array_equal(sa.acti_level, sb.acti_level)
        ta, tb = a.stats(), s.stats()
        assert (ta.cell_updates, ta.n_substeps, ta.n_splits, ta.n_unsplits, ta.tree_size) == \
            (tb.cell_updates, tb.n_substeps, tb.n_splits, tb.n_unsplits, tb.tree_size)
    for s in together + alone:
        s.close()


def test_lockstep_batch_multiphase_matches_reference(tmp_path):
    """Two five-equation trees of different sizes in one dg_batch against the reference solver."""
    trees = [cases.shock_drop(base_level=3, levels=2), cases.shock_drop(base_level=4, levels=1)]
    solvers = [Solver(c) for c in trees]
    b = Batch(solvers)
    for _ in range(2):
        assert not any(b.step())
    b.close()
    for k, (s, c) in enumerate(zip(solvers, trees)):
        path = str(tmp_path / f"m{k}.case")
        write_case(c, path)
        run_reference(path, str(tmp_path / f"m{k}"), 2, [2])
        ref = read_snapshot(str(tmp_path / f"m{k}_2.snap"))
        rep = compare(ref, s.active_cells(), c.params.side_length)
        assert rep.ok(1e-10), f"tree {k}: {rep}"
        s.close()
