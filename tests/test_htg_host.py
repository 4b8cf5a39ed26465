"""HTG writer (dacti_b200/htg.py) against the oracle's restatement of DACTI's htg_writer.

The oracle (oracle/htg_writer_ref.py) replays the reference's cursor walk, with global indices in
creation order and a depth-first breadth-first map. The product walks the node table level by level.
Both read the same node tables:
- tables that the reference integrator itself dumps (oracle/_ref runner, --nodes) after steps with
  regrid and garbage collection;
- host-built initial trees with inactive leaves;
- a hand-written tree whose file content is spelled out below.
No GPU needed.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, run_reference
from dacti_b200 import cases
from dacti_b200.casefile import read_snapshot
from dacti_b200.htg import NodeTable, hyper_tree, read_htg, write_frame, write_htg
from oracle.htg_writer_ref import read_nodes, reference_htg


def _table(d: dict) -> NodeTable:
    return NodeTable(d["dims"], d["parent"], d["children"], d["level"], d["flags"], d["p"], d["meta"])


def _same_as_reference(nodes: NodeTable, root: int, ref_nodes: NodeTable = None, extent: float = 1.0):
    r = ref_nodes or nodes
    desc, per_depth, mask, data = reference_htg(r.dims, r.parent, r.children, r.level, r.flags, r.p, r.meta, root)
    ht = hyper_tree(nodes, extent)
    assert ht.descriptor.tolist() == desc
    assert ht.vertices_per_level.tolist() == per_depth
    assert ht.mask.tolist() == mask
    for name, vals in data.items():
        got = ht.cell_data[name]
        want = np.array([0.0 if v is None else v for v in vals])
        assert np.array_equal(got, want), name
        assert all(got[k] == 0.0 for k, v in enumerate(vals) if v is None)
    return ht


def test_hand_tree_file_content(tmp_path):
    # 2D: root (slot 1) split; its child 1 (slot 3) split again; slot 7 is an inactive leaf
    C = 4
    n = 10
    parent = np.array([0, 0, 1, 1, 1, 1, 3, 3, 3, 3], np.int32)
    children = np.zeros((n, C), np.int32)
    children[1] = [2, 3, 4, 5]
    children[3] = [6, 7, 8, 9]
    level = np.array([0, 0, 1, 1, 1, 1, 2, 2, 2, 2], np.int32)
    flags = np.full(n, 3, np.uint32)
    flags[0] = 0
    flags[1] = flags[3] = 2
    flags[7] = 1
    p = np.arange(n, dtype=np.float64)[:, None] * np.array([[1.0, 10.0]])
    meta = np.tile([[2.0, 0.5, 1e-3, 0.25]], (n, 1))
    nodes = NodeTable(2, parent, children, level, flags, p, meta)
    ht = _same_as_reference(nodes, 1, extent=2.0)
    assert ht.descriptor.tolist() == [True, False, True, False, False]
    assert ht.vertices_per_level.tolist() == [1, 4, 4]
    assert ht.slots.tolist() == [1, 2, 3, 4, 5, 6, 7, 8, 9]
    assert ht.mask.astype(int).tolist() == [0, 0, 0, 0, 0, 0, 1, 0, 0]
    assert ht.cell_data["p_0"].tolist() == [0, 2, 0, 4, 5, 6, 7, 8, 9]
    assert ht.cell_data["acti_level"].tolist() == [0, 2, 0, 2, 2, 2, 2, 2, 2]
    for fmt in ("ascii", "binary"):
        path = str(tmp_path / f"hand_{fmt}.htg")
        write_htg(path, ht, fmt)
        back = read_htg(path)
        assert back["Descriptor"].astype(int).tolist() == [1, 0, 1, 0, 0]
        assert back["NbVerticesByLevel"].tolist() == [1, 4, 4]
        assert back["Mask"].astype(int).tolist() == [0, 0, 0, 0, 0, 0, 1, 0, 0]
        assert back["p_1"].tolist() == [0, 20, 0, 40, 50, 60, 70, 80, 90]
        # the base cell spans -+active_size[0]/2 on every axis, two values per axis also in 2D
        for axis in "XYZ":
            assert back[f"{axis}Coordinates"].tolist() == [-1.0, 1.0]
        assert back["NumberOfLevels"].tolist() == [3] and back["NumberOfVertices"].tolist() == [9]
        text = open(path).read()
        assert 'Dimensions="2 2 1"' in text and 'BranchFactor="2"' in text
    # binary Bit arrays: first vertex in the most significant bit of the first byte
    import base64
    text = open(str(tmp_path / "hand_binary.htg")).read()
    body = text.split('Name="Mask" NumberOfTuples="9" format="binary">')[1].split("<")[0]
    raw = base64.b64decode(body)
    assert int(np.frombuffer(raw[:8], np.uint64)[0]) == 2
    assert raw[8:] == bytes([0b00000010, 0b00000000])


def test_root_leaf_tree():
    # a single root leaf: one vertex, no descriptor bits, nothing written for the root
    nodes = NodeTable(3, np.zeros(2, np.int32), np.zeros((2, 8), np.int32), np.zeros(2, np.int32),
                      np.array([0, 3], np.uint32), np.ones((2, 5)), np.ones((2, 4)))
    ht = _same_as_reference(nodes, 1)
    assert ht.n_vertices == 1 and ht.n_levels == 1 and ht.descriptor.size == 0
    assert ht.cell_data["p_0"].tolist() == [0.0] and not ht.mask[0]


@pytest.mark.parametrize("name,steps,checks", [("euler2", 6, [2, 6]), ("multi2", 4, [0, 4]), ("euler3", 2, [2]),
                                               ("ns2_walls", 10, [10]), ("euler2_open_a", 10, [10]),
                                               ("euler2_periodic", 6, [6]), ("multi3", 2, [2]), ("ns3", 4, [4])])
def test_reference_node_tables(name, steps, checks, tmp_path):
    """Node tables that DACTI's integrator dumps after steps (regrid, garbage slots) give the same hyper
    tree through both walks, its unmasked leaves are exactly the snapshot's active cells, and the file
    reads back unchanged."""
    run_reference(os.path.join(GOLDEN, f"{name}.case"), str(tmp_path / name), steps, checks, extra=("--nodes",))
    for k in checks:
        d = read_nodes(str(tmp_path / f"{name}_{k}.nodes"))
        nodes = _table(d)
        ht = _same_as_reference(nodes, d["root"])
        snap = read_snapshot(str(tmp_path / f"{name}_{k}.snap"))
        leaf = (nodes.flags[ht.slots] & 1) != 0
        shown = leaf & ~ht.mask
        shown[0] = shown[0] and ht.n_vertices > 1
        assert int(shown.sum()) == snap.n
        got = np.sort(ht.cell_data["p_0"][shown])
        assert np.array_equal(got, np.sort(snap.p[:, 0]))
        path = write_frame(str(tmp_path / "out"), name, k, nodes, 1.0)
        assert path.endswith(f"{name}_{k:04d}.htg")
        back = read_htg(path)
        assert np.array_equal(back["Descriptor"], ht.descriptor)
        assert np.array_equal(back["Mask"], ht.mask)
        for q in range(d["E"]):
            assert np.array_equal(back[f"p_{q}"], ht.cell_data[f"p_{q}"])
        assert np.array_equal(back["cfl"], ht.cell_data["cfl"])


def test_slot_order_is_free(tmp_path):
    """A re-sorted slot order (as the device's Morton re-sort leaves it) writes the same tree."""
    run_reference(os.path.join(GOLDEN, "euler2.case"), str(tmp_path / "e"), 6, [6], extra=("--nodes",))
    d = read_nodes(str(tmp_path / "e_6.nodes"))
    nodes = _table(d)
    rng = np.random.default_rng(5)
    n = nodes.n
    perm = np.concatenate([[0], 1 + rng.permutation(n - 1)])   # new slot k holds old slot perm[k]
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    shuffled = NodeTable(2, inv[nodes.parent[perm]].astype(np.int32), inv[nodes.children[perm]].astype(np.int32),
                         nodes.level[perm], nodes.flags[perm], nodes.p[perm], nodes.meta[perm])
    a, b = hyper_tree(nodes, 1.0), hyper_tree(shuffled, 1.0)
    assert np.array_equal(a.descriptor, b.descriptor) and np.array_equal(a.mask, b.mask)
    assert np.array_equal(inv[a.slots], b.slots)
    for name in a.cell_data:
        assert np.array_equal(a.cell_data[name], b.cell_data[name])


def test_host_tree_with_inactive_leaves():
    c = cases.cylinder_ns(base_level=4, levels=2)
    t = c.tree
    meta = np.zeros((t.n_nodes, 4))
    nodes = NodeTable(2, t.parent, t.children, t.level, t.flags, t.p, meta)
    ht = _same_as_reference(nodes, 1, extent=40.0)
    inactive_leaves = int((((t.flags & 1) != 0) & ((t.flags & 2) == 0) & ((t.flags & 4) == 0)).sum())
    assert int(ht.mask.sum()) == inactive_leaves > 0


def test_bad_tables_raise():
    nodes = NodeTable(2, np.zeros(3, np.int32), np.zeros((3, 4), np.int32), np.zeros(3, np.int32),
                      np.array([0, 2, 2], np.uint32), np.zeros((3, 4)), np.zeros((3, 4)))
    with pytest.raises(ValueError):
        hyper_tree(nodes, 1.0)       # two live level-0 slots
    nodes.level[2] = 1
    with pytest.raises(ValueError):
        hyper_tree(nodes, 1.0)       # root subdivided with null child slots
    with pytest.raises(ValueError):
        write_htg("/dev/null", hyper_tree(NodeTable(2, np.zeros(2, np.int32), np.zeros((2, 4), np.int32),
                                                    np.zeros(2, np.int32), np.array([0, 3], np.uint32),
                                                    np.zeros((2, 4)), np.zeros((2, 4))), 1.0), fmt="xml")
