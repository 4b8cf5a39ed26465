"""Headless HyperTreeGrid output, as DACTI's htg_writer writes it (driver/io/htg_writer.hpp:17-195).

The reference builds a vtkHyperTreeGrid of one hyper tree (branch factor 2, a base grid of one cell)
by walking Integrator::get_nodes(): every non-leaf node is subdivided, level by level, and each child
of a subdivided node gets cell values when it is a leaf (htg_writer.hpp:117-162):
- p_0 .. p_{E-1}: the leaf's primitive state Cell::get_p() (cell.hpp:45-47);
- acti_level, error, max_dt, cfl: Node::get_metadata() (node.hpp:56-58);
- mask: set on inactive leaves (hidden), clear elsewhere.
Nothing is ever written for a non-leaf vertex or for the root, so those values are indeterminate in
the reference's files; they are 0 here. The base cell spans -+active_size[0]/2 along every axis, the
y and z extents included (htg_writer.hpp:51-61), and each coordinate array has two values, also in 2D.
The writer's `injections` (observer fields) are accepted and not written, as in the reference.

VTK is not needed: the file is the XML HyperTreeGrid layout that vtkXMLHyperTreeGridReader reads
(file version 1.0: one <Tree> element holding its Descriptor, NbVerticesByLevel, Mask and CellData).
The hyper tree is stored in breadth-first order: vertex k of depth d follows all of depth d - 1, and
the children of one vertex are consecutive in child order (child c has bit d of c set when it lies on
the positive side along dimension d, the reference's Children order, passed to ToChild unchanged).
Descriptor holds one bit per vertex above the deepest level (1 = subdivided); NbVerticesByLevel the
vertex count per depth; Mask one bit per vertex; every CellData array one value per vertex.
Arrays are written as ASCII or as base64 inline binary (UInt64 byte-count header; Bit arrays packed
eight to a byte, first vertex in the most significant bit, as vtkBitArray stores them).
"""
from __future__ import annotations

import base64
import os
from dataclasses import dataclass
from typing import Dict, List

import numpy as np

F_LEAF, F_ACTIVE, F_GARBAGE = 1, 2, 4
META_NAMES = ("acti_level", "error", "max_dt", "cfl")


@dataclass
class NodeTable:
    """The node slots of a tree, one row per slot (Integrator::get_nodes, integrator.hpp:165).

    parent (n,), children (n, 2^D), level (n,), flags (n,) with bits F_LEAF, F_ACTIVE, F_GARBAGE,
    p (n, E) and meta (n, 4) = {acti_level, error, max_dt, cfl}. Slot order is free: the hyper tree
    is walked from the root through the children."""
    dims: int
    parent: np.ndarray
    children: np.ndarray
    level: np.ndarray
    flags: np.ndarray
    p: np.ndarray
    meta: np.ndarray

    @property
    def n(self) -> int:
        return int(self.parent.shape[0])

    def root(self) -> int:
        live = np.nonzero((self.level == 0) & ((self.flags & F_GARBAGE) == 0))[0]
        live = live[live != 0]
        if live.size != 1:
            raise ValueError(f"expected one root (a live level-0 slot other than the null slot 0), found {live.size}")
        return int(live[0])


@dataclass
class HyperTree:
    """One hyper tree in breadth-first order, as the HTG file stores it."""
    dims: int
    extent: float                 # active_size[0]: the base cell spans -+extent/2 on every axis
    descriptor: np.ndarray        # bool, one per vertex above the deepest level
    vertices_per_level: np.ndarray
    mask: np.ndarray              # bool, one per vertex
    cell_data: Dict[str, np.ndarray]
    slots: np.ndarray             # node slot of each vertex (not written; for callers and checks)

    @property
    def n_vertices(self) -> int:
        return int(self.mask.shape[0])

    @property
    def n_levels(self) -> int:
        return int(self.vertices_per_level.shape[0])


def hyper_tree(nodes: NodeTable, active_size0: float) -> HyperTree:
    """Breadth-first hyper tree of `nodes`, with the reference writer's values and mask."""
    C = 1 << nodes.dims
    root = nodes.root()
    leaf = (nodes.flags & F_LEAF) != 0
    depth_slots: List[np.ndarray] = [np.array([root], np.int64)]
    bits: List[np.ndarray] = []
    while True:
        cur = depth_slots[-1]
        refined = ~leaf[cur]
        if not refined.any():
            break
        bits.append(refined)
        kids = nodes.children[cur[refined]].astype(np.int64).reshape(-1)
        if (kids <= 0).any() or (kids >= nodes.n).any():
            raise ValueError("a subdivided node has a child slot outside the table")
        depth_slots.append(kids)
        if len(depth_slots) > 64:
            raise ValueError("tree deeper than 64 levels (a cycle in the child links?)")
    slots = np.concatenate(depth_slots)
    written = leaf[slots]
    written[0] = False                      # the root is never a child: nothing is written for it
    mask = written & ((nodes.flags[slots] & F_ACTIVE) == 0)
    E = nodes.p.shape[1]
    data: Dict[str, np.ndarray] = {}
    for q in range(E):
        data[f"p_{q}"] = np.where(written, nodes.p[slots, q], 0.0)
    for j, name in enumerate(META_NAMES):
        data[name] = np.where(written, nodes.meta[slots, j], 0.0)
    return HyperTree(
        dims=nodes.dims, extent=float(active_size0),
        descriptor=np.concatenate(bits) if bits else np.zeros(0, bool),
        vertices_per_level=np.array([s.size for s in depth_slots], np.int64),
        mask=mask, cell_data=data, slots=slots,
    )


def _values(a: np.ndarray, typ: str, fmt: str) -> bytes:
    if fmt == "ascii":
        if typ == "Bit" or typ == "Int64":
            return " ".join(str(int(v)) for v in a).encode("ascii")
        return " ".join(repr(float(v)) for v in a).encode("ascii")
    if typ == "Bit":
        raw = np.packbits(a.astype(np.uint8), bitorder="big").tobytes()
    elif typ == "Int64":
        raw = np.ascontiguousarray(a, "<i8").tobytes()
    else:
        raw = np.ascontiguousarray(a, "<f8").tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw)


def _array(f, name: str, a: np.ndarray, typ: str, fmt: str, indent: str) -> None:
    f.write(f'{indent}<DataArray type="{typ}" Name="{name}" NumberOfTuples="{a.shape[0]}" format="{fmt}">'
            .encode("ascii"))
    f.write(_values(a, typ, fmt))
    f.write(b"</DataArray>\n")


def write_htg(path: str, ht: HyperTree, fmt: str = "binary") -> None:
    """Writes `ht` as an XML HyperTreeGrid file (`fmt` "binary" or "ascii")."""
    if fmt not in ("binary", "ascii"):
        raise ValueError("fmt is 'binary' or 'ascii'")
    dims = {1: "2 1 1", 2: "2 2 1", 3: "2 2 2"}[ht.dims]
    h = 0.5 * ht.extent
    base = np.array([-h, h])
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "wb") as f:
        f.write(('<?xml version="1.0"?>\n'
                 '<VTKFile type="HyperTreeGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n'
                 f'  <HyperTreeGrid BranchFactor="2" TransposedRootIndexing="0" Dimensions="{dims}">\n'
                 "    <Grid>\n").encode("ascii"))
        for axis in "XYZ":
            _array(f, f"{axis}Coordinates", base, "Float64", fmt, "      ")
        f.write(("    </Grid>\n    <Trees>\n"
                 f'      <Tree Index="0" NumberOfLevels="{ht.n_levels}" NumberOfVertices="{ht.n_vertices}">\n')
                .encode("ascii"))
        _array(f, "Descriptor", ht.descriptor, "Bit", fmt, "        ")
        _array(f, "NbVerticesByLevel", ht.vertices_per_level, "Int64", fmt, "        ")
        _array(f, "Mask", ht.mask, "Bit", fmt, "        ")
        f.write(b"        <CellData>\n")
        for name, v in ht.cell_data.items():
            _array(f, name, v, "Float64", fmt, "          ")
        f.write(b"        </CellData>\n      </Tree>\n    </Trees>\n  </HyperTreeGrid>\n</VTKFile>\n")


def write_frame(out_dir: str, name: str, frame: int, nodes: NodeTable, active_size0: float,
                fmt: str = "binary", injections=None, injection_names=None) -> str:
    """htg_writer::write_data: `<out_dir>/<name>_<frame:04>.htg` (htg_writer.hpp:169); observer fields
    (`injections`) are not written, as in the reference."""
    path = os.path.join(out_dir, f"{name}_{frame:04d}.htg")
    write_htg(path, hyper_tree(nodes, active_size0), fmt)
    return path


def read_htg(path: str) -> Dict[str, np.ndarray]:
    """Decodes every named DataArray of a file written by write_htg, plus the Tree attributes
    (for checks and tests)."""
    import re
    text = open(path).read()
    out: Dict[str, np.ndarray] = {}
    m = re.search(r'<Tree Index="0" NumberOfLevels="(\d+)" NumberOfVertices="(\d+)">', text)
    if m:
        out["NumberOfLevels"] = np.array([int(m.group(1))])
        out["NumberOfVertices"] = np.array([int(m.group(2))])
    for m in re.finditer(r'<DataArray type="(\w+)" Name="([^"]+)" NumberOfTuples="(\d+)" format="(\w+)">([^<]*)'
                         r"</DataArray>", text):
        typ, name, n, fmt, body = m.group(1), m.group(2), int(m.group(3)), m.group(4), m.group(5)
        if fmt == "ascii":
            toks = body.split()
            if typ == "Float64":
                a = np.array([float(t) for t in toks], np.float64)
            else:
                a = np.array([int(t) for t in toks], np.int64)
        else:
            raw = base64.b64decode(body)
            nbytes = int(np.frombuffer(raw[:8], np.uint64)[0])
            raw = raw[8:8 + nbytes]
            if typ == "Bit":
                a = np.unpackbits(np.frombuffer(raw, np.uint8), bitorder="big")[:n].astype(np.int64)
            else:
                a = np.frombuffer(raw, {"Int64": "<i8", "Float64": "<f8"}[typ]).copy()
        if a.shape[0] != n:
            raise ValueError(f"{name}: {a.shape[0]} values, NumberOfTuples says {n}")
        out[name] = a.astype(bool) if typ == "Bit" else a
    return out
