"""Host-side tree builder and case-file format (no GPU)."""
import numpy as np

from dacti_b200 import cases
from dacti_b200.casefile import read_case, write_case
from dacti_b200.models import F_ACTIVE, F_LEAF, ModelId


def _check_tree(case):
    t = case.tree
    D = t.shape.dims
    side = case.params.side_length
    leaf = (t.flags & F_LEAF) != 0
    internal = np.nonzero(~leaf)[0]
    internal = internal[internal > 0]
    for i in internal:
        kids = t.children[i]
        assert (kids > 0).all()
        assert (t.parent[kids] == i).all()
        assert (t.level[kids] == t.level[i] + 1).all()
        size = side * 0.5 ** t.level[i]
        for c, k in enumerate(kids):
            q = np.array([1.0 if (c >> d) & 1 else -1.0 for d in range(D)])
            # Domain::split: child.center = parent.center + 0.25 * parent.size * quadrant(i)
            assert np.array_equal(t.center[k], t.center[i] + (0.25 * size) * q)
    assert t.level[1] == 0 and t.parent[1] == 0


def test_lax_liu_tree_is_uniform_base_grid():
    c = cases.lax_liu3(base_level=4, levels=2)
    _check_tree(c)
    m = c.tree.leaf_mask()
    assert m.sum() == 16 * 16
    assert (c.tree.level[m] == 4).all()
    # quadrant states
    p = c.tree.p[m]
    ctr = c.tree.center[m]
    tr = (ctr[:, 0] > 0) & (ctr[:, 1] > 0)
    assert np.allclose(p[tr], [1.5, 0, 0, 1.5])
    # every boundary face of the base grid carries a domain boundary
    nb = (c.tree.bc[m] >= 0).sum()
    assert nb == 4 * 16


def test_shock_drop_tree_refines_drop_and_shock():
    c = cases.shock_drop(dims=3, base_level=3, levels=2)
    _check_tree(c)
    t = c.tree
    m = t.leaf_mask()
    assert (t.level[m] <= 5).all() and (t.level[m] == 5).any()
    alpha = t.p[m, t.shape.ia]
    assert alpha.max() > 0.5 and alpha.min() == 0.0
    # inactive cells lie outside the 8 x 4 x 4 mm box
    inactive = ((t.flags & F_LEAF) != 0) & ((t.flags & F_ACTIVE) == 0)
    inactive[0] = False
    assert (np.abs(t.center[inactive, 1:]) > 2e-3).any(axis=1).all()


def test_periodic_case_has_no_boundaries():
    c = cases.periodic_blob(base_level=3, levels=1)
    assert len(c.tree.bcs) == 0
    assert (c.tree.bc == -1).all()


def test_case_file_roundtrip(tmp_path):
    for c in (cases.lax_liu3(base_level=3, levels=1),
              cases.lax_liu3(base_level=3, levels=1, model=ModelId.NAVIER_STOKES, mu=1e-3, prandtl=0.7),
              cases.shock_drop(dims=2, base_level=3, levels=1)):
        a = tmp_path / "a.case"
        b = tmp_path / "b.case"
        write_case(c, str(a))
        write_case(read_case(str(a)), str(b))
        assert a.read_bytes() == b.read_bytes()


def test_prune_inactive_keeps_every_active_leaf_and_counts_the_rest():
    """prune_inactive drops exactly the subtrees without an active leaf: the active leaves, their
    ancestors and their states stay, links stay consistent, and the dropped slots are counted."""
    import numpy as np

    from dacti_b200 import cases
    from dacti_b200.casefile import prune_inactive

    for case in (cases.shock_drop(base_level=4, levels=2), cases.cylinder_ns(mach=0.3, base_level=4, levels=2)):
        t, p = case.tree, prune_inactive(case)
        q = p.tree
        assert p.params.pruned_nodes == t.n_nodes - q.n_nodes > 0
        a, b = t.leaf_mask(), q.leaf_mask()
        assert a.sum() == b.sum()
        oa, ob = np.lexsort(t.center[a].T), np.lexsort(q.center[b].T)
        assert np.array_equal(t.center[a][oa], q.center[b][ob]) and np.array_equal(t.p[a][oa], q.p[b][ob])
        assert np.array_equal(t.bc[a][oa], q.bc[b][ob]) and np.array_equal(t.level[a][oa], q.level[b][ob])
        # every kept node's children point back at it; the root's parent is the null slot
        assert q.parent[1] == 0
        for c in range(q.children.shape[1]):
            ch = q.children[:, c]
            live = ch > 0
            assert np.array_equal(q.parent[ch[live]], np.nonzero(live)[0])
        assert p.params.param_vector()[29] == p.params.pruned_nodes
