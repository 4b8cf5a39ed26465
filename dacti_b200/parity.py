"""Snapshot comparison used by the parity tests and the bench's accuracy check.

Two snapshots agree on refinement decisions when they hold the same set of cells, keyed by
(tree level, integer cell coordinates), with the same ACTI level per cell; conserved fields are
compared by relative L1 norm per component.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .casefile import Snapshot, cell_coords


@dataclass
class ParityReport:
    n_ref: int
    n_gpu: int
    same_cells: bool
    acti_mismatch: int
    rel_l1: np.ndarray  # per conserved component
    max_abs_t: float
    only_ref: int
    only_gpu: int

    @property
    def max_rel_l1(self) -> float:
        return float(np.max(self.rel_l1)) if self.rel_l1.size else 0.0

    def ok(self, tol: float) -> bool:
        return self.same_cells and self.acti_mismatch == 0 and self.max_rel_l1 <= tol

    def __str__(self) -> str:
        return (f"cells ref={self.n_ref} gpu={self.n_gpu} same={self.same_cells} only_ref={self.only_ref} "
                f"only_gpu={self.only_gpu} acti_mismatch={self.acti_mismatch} max_rel_l1={self.max_rel_l1:.3e} "
                f"rel_l1={np.array2string(self.rel_l1, precision=2)} max|dt|={self.max_abs_t:.2e}")


def _keys(s: Snapshot, side: float) -> np.ndarray:
    c = cell_coords(s.center, s.tree_level, side)
    k = s.tree_level.astype(np.int64)
    for d in range(s.dims):
        k = k * (1 << 21) + c[:, d]
    return k


def compare(ref: Snapshot, gpu: Snapshot, side_length: float) -> ParityReport:
    kr, kg = _keys(ref, side_length), _keys(gpu, side_length)
    orr, og = np.argsort(kr), np.argsort(kg)
    kr_s, kg_s = kr[orr], kg[og]
    common, ir, ig = np.intersect1d(kr_s, kg_s, assume_unique=True, return_indices=True)
    same = ref.n == gpu.n and common.size == ref.n
    a = orr[ir]
    b = og[ig]
    acti_mm = int(np.count_nonzero(ref.acti_level[a] != gpu.acti_level[b]))
    ur, ug = ref.u[a], gpu.u[b]
    denom = np.abs(ur).sum(axis=0)
    denom = np.where(denom > 0, denom, 1.0)
    rel = np.abs(ur - ug).sum(axis=0) / denom
    dt = float(np.max(np.abs(ref.t[a] - gpu.t[b]))) if a.size else 0.0
    return ParityReport(ref.n, gpu.n, bool(same), acti_mm, rel, dt, int(ref.n - common.size),
                        int(gpu.n - common.size))
