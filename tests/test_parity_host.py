"""The snapshot comparison behind every parity test (dacti_b200.parity.compare), on synthetic cell sets:
order does not matter, a moved or missing cell breaks `same_cells`, ACTI-level and state differences are
counted per component."""
import numpy as np

from dacti_b200.casefile import Snapshot
from dacti_b200.parity import compare

SIDE = 1.0


def _uniform(level=3, seed=0):
    n1 = 1 << level
    idx = np.stack(np.meshgrid(np.arange(n1), np.arange(n1), indexing="ij"), -1).reshape(-1, 2)
    center = (idx + 0.5) / n1 * SIDE - 0.5 * SIDE
    n = center.shape[0]
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.5, 2.0, (n, 4))
    z = np.zeros(n)
    return Snapshot(2, 4, 1, 1, n, n, 0.1, 0.1, float(n), np.full(n, level, np.int32), np.zeros(n, np.int32),
                    center, np.full(n, 0.1), u, u.copy(), z, z, z)


def _permuted(s, order):
    return Snapshot(s.dims, s.E, s.step, s.n_substeps, s.tree_size, s.n_in_clusters, s.time, s.global_dt,
                    s.updates, s.tree_level[order], s.acti_level[order], s.center[order], s.t[order],
                    s.u[order], s.p[order], s.error[order], s.max_dt[order], s.cfl[order])


def test_identical_sets_in_any_order_agree_exactly():
    a = _uniform()
    b = _permuted(a, np.random.default_rng(1).permutation(a.n))
    rep = compare(a, b, SIDE)
    assert rep.same_cells and rep.acti_mismatch == 0 and rep.max_rel_l1 == 0.0 and rep.ok(0.0)


def test_state_difference_is_a_relative_l1_per_component():
    a = _uniform()
    b = _permuted(a, np.arange(a.n))
    b.u = a.u.copy()
    b.u[5, 2] += 1e-3
    rep = compare(a, b, SIDE)
    assert rep.same_cells and rep.rel_l1[0] == 0.0 and rep.rel_l1[1] == 0.0 and rep.rel_l1[3] == 0.0
    assert np.isclose(rep.rel_l1[2], 1e-3 / np.abs(a.u[:, 2]).sum())
    assert rep.ok(1e-3) and not rep.ok(1e-12)


def test_acti_level_and_cell_set_differences_fail():
    a = _uniform()
    b = _permuted(a, np.arange(a.n))
    b.acti_level = a.acti_level.copy()
    b.acti_level[3] = 1
    rep = compare(a, b, SIDE)
    assert rep.same_cells and rep.acti_mismatch == 1 and not rep.ok(1.0)
    # one cell replaced by a cell one level finer at the same corner: the sets differ
    c = _permuted(a, np.arange(a.n))
    c.tree_level = a.tree_level.copy()
    c.center = a.center.copy()
    c.tree_level[0] = a.tree_level[0] + 1
    c.center[0] = a.center[0] - 0.25 * SIDE / (1 << int(a.tree_level[0]))
    rep = compare(a, c, SIDE)
    assert not rep.same_cells and rep.only_ref == 1 and rep.only_gpu == 1 and not rep.ok(1.0)
