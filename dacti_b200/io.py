"""Headless VTU output of the active cells, as DACTI's vtu_writer writes it (driver/io/vtu_writer.hpp).

One VTK_VOXEL per active cell with its 8 vertices at centre +- size/2 (in 2D the cell gets a z extent
of 0.01); point data p_0..p_{E-1} is the cell's linear reconstruction Cell::get_p(x, t) = p + slope (x -
centre) at each vertex (integrator/cell.hpp:23-31); cell data k_0..k_{P-1}, the metadata acti_level,
error, max_dt, cfl, and any extra per-cell fields. Written as XML with base64 inline binary arrays
(UInt64 byte-count headers), which ParaView and VTK read; VTK itself is not needed.
"""
from __future__ import annotations

import base64
import os
from typing import Dict, Optional

import numpy as np

from .casefile import Snapshot

VTK_VOXEL = 11
META_NAMES = ("acti_level", "error", "max_dt", "cfl")


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")


def _array(name: Optional[str], a: np.ndarray, comps: int = 1) -> str:
    vtk = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8"}[a.dtype]
    nm = f' Name="{name}"' if name else ""
    return (f'<DataArray type="{vtk}"{nm} NumberOfComponents="{comps}" format="binary">'
            f"{_b64(a)}</DataArray>\n")


def voxel_points(snap: Snapshot, side_length: float) -> np.ndarray:
    """(n, 8, 3) vertex coordinates, vertex j at quadrant j (bit d set: +size/2 along d)."""
    n, D = snap.n, snap.dims
    size = side_length * 0.5 ** snap.tree_level.astype(np.float64)
    c3 = np.zeros((n, 3))
    c3[:, :D] = snap.center
    s3 = np.full((n, 3), 0.01)
    s3[:, :D] = size[:, None]
    q = np.array([[1.0 if (j >> d) & 1 else -1.0 for d in range(3)] for j in range(8)])
    return c3[:, None, :] + 0.5 * q[None, :, :] * s3[:, None, :]


def write_vtu(path: str, snap: Snapshot, slopes: np.ndarray, side_length: float,
              fields: Optional[Dict[str, np.ndarray]] = None) -> None:
    """Writes the active cells of `snap` (with their slopes, shape (n, D, E)) to `path`."""
    n, D, E = snap.n, snap.dims, snap.E
    pts = voxel_points(snap, side_length)                       # (n, 8, 3)
    dx = pts[:, :, :D] - snap.center[:, None, :]                # (n, 8, D)
    pv = snap.p[:, None, :] + np.einsum("nvd,nde->nve", dx, slopes[:n])
    conn = np.arange(8 * n, dtype=np.int64)
    offsets = 8 * np.arange(1, n + 1, dtype=np.int64)
    types = np.full(n, VTK_VOXEL, np.uint8)
    meta = {"acti_level": snap.acti_level.astype(np.float64), "error": snap.error, "max_dt": snap.max_dt,
            "cfl": snap.cfl}
    out = ['<?xml version="1.0"?>\n',
           '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" header_type="UInt64">\n',
           "<UnstructuredGrid>\n", f'<Piece NumberOfPoints="{8 * n}" NumberOfCells="{n}">\n',
           "<Points>\n", _array(None, pts.reshape(-1, 3), 3), "</Points>\n",
           "<Cells>\n", _array("connectivity", conn), _array("offsets", offsets), _array("types", types), "</Cells>\n",
           "<PointData>\n"]
    for q in range(E):
        out.append(_array(f"p_{q}", np.ascontiguousarray(pv[:, :, q]).reshape(-1)))
    out.append("</PointData>\n<CellData>\n")
    if snap.k is not None:
        for q in range(snap.k.shape[1]):
            out.append(_array(f"k_{q}", np.ascontiguousarray(snap.k[:, q])))
    for name in META_NAMES:
        out.append(_array(name, np.ascontiguousarray(meta[name], np.float64)))
    for name, v in (fields or {}).items():
        out.append(_array(name, np.ascontiguousarray(v, np.float64)))
    out.append("</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("".join(out))


def read_vtu_arrays(path: str) -> Dict[str, np.ndarray]:
    """Decodes every named DataArray of a file written by write_vtu (for checks and tests)."""
    import re
    text = open(path).read()
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: Name="([^"]+)")? NumberOfComponents="(\d+)" format="binary">'
                         r"([^<]*)</DataArray>", text):
        typ, name, comps, data = m.group(1), m.group(2) or "Points", int(m.group(3)), m.group(4)
        raw = base64.b64decode(data)
        nbytes = int(np.frombuffer(raw[:8], np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[typ]
        a = np.frombuffer(raw[8:8 + nbytes], dt)
        out[name] = a.reshape(-1, comps) if comps > 1 else a
    return out
