"""Accuracy of one solution against another on possibly different adaptive meshes.

Both solutions are projected conservatively onto the uniform grid of one tree level: a leaf finer
than that level adds its volume-weighted state to the covering cell, a coarser leaf fills every cell
it covers. The mixture density is the sum of the partial densities for the five-equation model
(model/multi.hpp:84) and rho itself for Euler/Navier-Stokes.
"""
from __future__ import annotations

import numpy as np

from .casefile import Snapshot, cell_coords


def project_uniform(snap: Snapshot, side: float, active, level: int) -> np.ndarray:
    """Conserved fields averaged onto the uniform grid of `level` over the active box: (cells, E)."""
    D, E = snap.dims, snap.E
    n_l = 1 << level
    h = side / n_l
    act = np.asarray(active, np.float64)[:D]
    a0 = np.rint((side - act) / 2.0 / h).astype(np.int64)
    na = np.rint(act / h).astype(np.int64)
    out = np.zeros((int(np.prod(na)), E))
    lv = snap.tree_level.astype(np.int64)
    coords = cell_coords(snap.center, lv, side)
    fine = lv >= level
    # finer leaves: volume fraction 2^{-D (lv - level)} of the coarse cell
    cf = (coords[fine] >> (lv[fine] - level)[:, None]) - a0
    wf = 0.5 ** (D * (lv[fine] - level))
    idx = np.ravel_multi_index(tuple(cf.T), tuple(na))
    np.add.at(out, idx, snap.u[fine] * wf[:, None])
    # coarser leaves cover 2^{D (level - lv)} uniform cells
    coarse = np.nonzero(~fine)[0]
    for k in np.unique(level - lv[coarse]):
        sel = coarse[(level - lv[coarse]) == k]
        lo = (coords[sel] << k) - a0
        off = np.stack(np.meshgrid(*[np.arange(1 << k)] * D, indexing="ij"), -1).reshape(-1, D)
        cells = (lo[:, None, :] + off[None, :, :]).reshape(-1, D)
        idx = np.ravel_multi_index(tuple(cells.T), tuple(na))
        np.add.at(out, idx, np.repeat(snap.u[sel], off.shape[0], axis=0))
    return out


def mixture_density(u: np.ndarray, model: int) -> np.ndarray:
    return u[:, 0] + u[:, 1] if model == 2 else u[:, 0]


def density_rel_l1(a: Snapshot, b: Snapshot, side: float, active, level: int, model: int) -> float:
    """sum |rho_a - rho_b| / sum |rho_b| on the uniform grid of `level` (b is the reference)."""
    ra = mixture_density(project_uniform(a, side, active, level), model)
    rb = mixture_density(project_uniform(b, side, active, level), model)
    return float(np.abs(ra - rb).sum() / np.abs(rb).sum())
