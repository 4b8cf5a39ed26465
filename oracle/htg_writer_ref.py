"""Oracle (test infrastructure, not the product): DACTI's HTG writer restated step by step.

What it restates:
- driver/io/htg_writer.hpp:100-162. The reference subdivides the hyper tree through a
  vtkHyperTreeGridNonOrientedCursor. It visits the non-leaf nodes of Integrator::get_nodes() level by
  level, in tree order (assign_to_split_node_sets, :176-183). For each one it walks from the root
  along the child indices found by get_path_to_root (:185-194), then calls SubdivideLeaf. Each new
  child gets the next global index, counted from SetGlobalIndexStart(root_index). Cell values and
  the mask are stored with InsertTuple1 at those global indices: values only for leaf children,
  mask false for every child, true for inactive leaf children, false for the root.
- VTK's vtkHyperTree::ComputeBreadthFirstOrderDescriptor. VTK 9.3 is the version the reference's
  CMakeLists.txt:26 asks for; VTK is not part of the reference tree and not installed here. The
  writer uses it to store the tree: a depth-first walk from the root appends each vertex to the list
  of its depth, and each vertex above the deepest level adds one "is subdivided" bit to its depth's
  descriptor. The file holds the per-depth lists one after another. Values are picked by global
  index through that breadth-first map.

Values that the reference never writes (non-leaf vertices and the root) come back as None here.
The product writer (dacti_b200/htg.py) computes the same tree with a level-by-level vectorised walk.
`read_nodes` reads the node table that oracle/ref/runner.cpp dumps with --nodes.
"""
from __future__ import annotations

import numpy as np

F_LEAF, F_ACTIVE, F_GARBAGE = 1, 2, 4


def read_nodes(path: str) -> dict:
    """A DGNODE01 file: header {D, E, n, root}, per node int32 parent, children[2^D], level, flags,
    then double p[E], metadata[4]."""
    buf = open(path, "rb").read()
    if buf[:8] != b"DGNODE01":
        raise ValueError("bad node-table magic")
    D, E, n, root = (int(x) for x in np.frombuffer(buf, np.int32, 4, 8))
    C = 1 << D
    rec = np.dtype([("i", "<i4", (3 + C,)), ("d", "<f8", (E + 4,))])
    r = np.frombuffer(buf, rec, n, 24)
    iv, dv = r["i"], r["d"]
    return dict(dims=D, E=E, root=root, parent=iv[:, 0].copy(), children=iv[:, 1:1 + C].copy(),
                level=iv[:, 1 + C].copy(), flags=iv[:, 2 + C].astype(np.uint32), p=dv[:, :E].copy(),
                meta=dv[:, E:].copy())


class _Vertex:
    __slots__ = ("gid", "children")

    def __init__(self, gid):
        self.gid = gid
        self.children = None


def reference_htg(dims, parent, children, level, flags, p, meta, root):
    """The hyper tree as the reference builds it and VTK stores it: (descriptor bits, vertices per
    depth, mask bits, {array name: values}) in breadth-first order, unwritten values None."""
    C = 1 << dims
    E = p.shape[1]
    n = len(parent)
    # htg_writer.hpp:114-115, 176-183: non-leaf nodes from the root index on, bucketed by tree level
    split_sets = {}
    for i in range(root, n):
        if not (flags[i] & F_LEAF):
            split_sets.setdefault(int(level[i]), []).append(i)
    top = _Vertex(root)          # SetGlobalIndexStart(root_index): the root's global index
    next_gid = root + 1
    values = {f"p_{q}": {} for q in range(E)}
    for name in ("acti_level", "error", "max_dt", "cfl"):
        values[name] = {}
    mask = {root: False}         # :103
    for lv in range(64):
        if lv not in split_sets:
            break
        for index in split_sets[lv]:
            # get_path_to_root (:185-194): child positions from the node up to the root
            path, child, par = [], index, int(parent[index])
            for _ in range(int(level[index]), 0, -1):
                row = list(children[par])
                path.append(row.index(child) if child in row else 0)   # Node::find_child returns 0 when absent
                child, par = par, int(parent[par])
            v = top
            for k in reversed(path):
                v = v.children[k]
            if v.children is not None:
                raise ValueError("node subdivided twice")
            v.children = []
            for c in range(C):                   # SubdivideLeaf: consecutive global indices
                v.children.append(_Vertex(next_gid))
                next_gid += 1
            for c in range(C):                   # :137-158
                node = int(children[index][c])
                gid = v.children[c].gid
                mask[gid] = False
                if flags[node] & F_LEAF:
                    for q in range(E):
                        values[f"p_{q}"][gid] = float(p[node][q])
                    for j, name in enumerate(("acti_level", "error", "max_dt", "cfl")):
                        values[name][gid] = float(meta[node][j])
                    if not (flags[node] & F_ACTIVE):
                        mask[gid] = True
    # ComputeBreadthFirstOrderDescriptor: depth-first walk appending to per-depth lists
    ids, bits = [], []

    def depth_of(v, d=0):
        return d if v.children is None else max(depth_of(c, d + 1) for c in v.children)

    n_levels = depth_of(top) + 1
    ids = [[] for _ in range(n_levels)]
    bits = [[] for _ in range(n_levels)]
    stack = [(top, 0)]
    while stack:
        v, d = stack.pop()
        ids[d].append(v.gid)
        if d + 1 < n_levels:
            bits[d].append(v.children is not None)
        if v.children is not None:
            for c in reversed(v.children):
                stack.append((c, d + 1))
    order = [g for lst in ids for g in lst]
    descriptor = [b for lst in bits for b in lst]
    per_depth = [len(lst) for lst in ids]
    mask_bf = [bool(mask.get(g, False)) for g in order]
    data = {name: [vals.get(g) for g in order] for name, vals in values.items()}
    return descriptor, per_depth, mask_bf, data
