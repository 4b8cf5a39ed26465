"""Learned regrid forecaster (no counterpart in the reference).

A small network (csrc/forecast.cu: n_in -> 64 -> 64 -> 1, trained with Adam on FP32 master weights,
predicting with BF16 weights) reads per-leaf features that the solver computes on the GPU
(`Solver.forecast_features`) and predicts whether the refinement indicator will fire at the leaf's
place `horizon` global steps ahead. Labels come from the solver's own later states: a leaf at step n
is positive when, at step n + horizon, its region holds a leaf whose indicator value exceeds the split
threshold or has been refined past the leaf's level, or lies inside a flagged coarser leaf.

The method without the network ("persistence") predicts that exactly the leaves flagged now stay
flagged; `scores` rates either against the labels. `run_with_forecast` drives the solver's regrid
with the network's predictions.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from .casefile import Snapshot, cell_coords
from .solver import DG_OK, DgError, Solver, load_library

_FP = ctypes.POINTER(ctypes.c_float)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, np.float32)


class Mlp:
    """dg_mlp: the forecaster network on the current device."""

    def __init__(self, n_in: int, seed: int = 1):
        self._lib = load_library()
        h = ctypes.c_void_p()
        self._check(self._lib.dg_mlp_create(n_in, seed, ctypes.byref(h)))
        self._h = h
        self.n_in = n_in
        n = ctypes.c_longlong(0)
        self._check(self._lib.dg_mlp_param_count(self._h, ctypes.byref(n)))
        self.n_params = n.value

    def _check(self, rc: int) -> None:
        if rc != DG_OK:
            raise DgError(rc, self._lib.dg_mlp_last_error().decode())

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        self._check(self._lib.dg_mlp_get_params(self._h, out.ctypes.data_as(_FP)))
        return out

    @params.setter
    def params(self, value) -> None:
        v = _f32(value)
        if v.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        self._check(self._lib.dg_mlp_set_params(self._h, v.ctypes.data_as(_FP)))

    def predict(self, x) -> np.ndarray:
        x = _f32(x).reshape(-1, self.n_in)
        out = np.zeros(x.shape[0], np.float32)
        self._check(self._lib.dg_mlp_predict(self._h, x.ctypes.data_as(_FP), x.shape[0], out.ctypes.data_as(_FP)))
        return out

    def loss_grad(self, x, y, pos_weight: float = 1.0):
        """(sum of the loss, sum of its gradient) over the samples, with the FP32 master weights."""
        x = _f32(x).reshape(-1, self.n_in)
        y = _f32(y).reshape(-1)
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_double(0.0)
        self._check(self._lib.dg_mlp_loss_grad(self._h, x.ctypes.data_as(_FP), y.ctypes.data_as(_FP), x.shape[0],
                                               pos_weight, g.ctypes.data_as(_FP), ctypes.byref(loss)))
        return loss.value, g

    def train(self, x, y, epochs: int = 20, batch: int = 1024, lr: float = 3e-3, pos_weight: float = 1.0,
              seed: int = 7) -> float:
        x = _f32(x).reshape(-1, self.n_in)
        y = _f32(y).reshape(-1)
        loss = ctypes.c_double(0.0)
        self._check(self._lib.dg_mlp_train(self._h, x.ctypes.data_as(_FP), y.ctypes.data_as(_FP), x.shape[0], epochs,
                                           batch, lr, pos_weight, seed, ctypes.byref(loss)))
        return loss.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dg_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _keys(level: np.ndarray, coords: np.ndarray) -> np.ndarray:
    """One integer per (level, cell coordinates): 4 bits of level and 20 bits per coordinate."""
    k = level.astype(np.uint64) << np.uint64(60)
    for d in range(coords.shape[1]):
        k |= coords[:, d].astype(np.uint64) << np.uint64(40 - 20 * d)
    return k


def flagged(snap: Snapshot, max_err: float) -> np.ndarray:
    """Leaves whose last indicator value calls for a split (impl/adaptive_refinement.hpp:16-94)."""
    return snap.error > max_err


def region_labels(now: Snapshot, future: Snapshot, side: float, max_err: float) -> np.ndarray:
    """For each leaf of `now`: whether, in `future`, its region holds a flagged leaf or a leaf finer
    than itself, or lies inside a flagged coarser leaf."""
    lf = future.tree_level.astype(np.int64)
    cf = cell_coords(future.center, lf, side)
    ff = flagged(future, max_err)
    pos = []
    for l in range(int(lf.max()) + 1 if lf.size else 0):
        # ancestors at level l of future leaves finer than l (refined there) or at l..: flagged
        finer = lf > l
        sel = finer | (ff & (lf >= l))
        if sel.any():
            shift = (lf[sel] - l).astype(np.int64)
            pos.append(_keys(np.full(sel.sum(), l), cf[sel] >> shift[:, None]))
    pos_keys = np.unique(np.concatenate(pos)) if pos else np.zeros(0, np.uint64)
    flag_keys = np.unique(_keys(lf[ff], cf[ff])) if ff.any() else np.zeros(0, np.uint64)
    ln = now.tree_level.astype(np.int64)
    cn = cell_coords(now.center, ln, side)
    lab = np.isin(_keys(ln, cn), pos_keys)
    for l in range(int(ln.max()) if ln.size else 0):
        coarser = ln > l
        if coarser.any():
            anc = _keys(np.full(coarser.sum(), l), cn[coarser] >> (ln[coarser] - l)[:, None])
            lab[np.nonzero(coarser)[0][np.isin(anc, flag_keys)]] = True
    return lab


@dataclass
class RunData:
    x: np.ndarray           # features of every (step, leaf) pair
    y: np.ndarray           # labels
    persistence: np.ndarray  # the method without the network: flagged now
    steps: int


def collect(case: Callable[[], object], steps: int, horizon: int) -> RunData:
    """Runs a case for `steps` global steps on the GPU, reading features and leaves after each, and
    labels every step n <= steps - horizon from step n + horizon."""
    s = Solver(case())
    max_err = float(s.params.error_threshold[1])
    feats, snaps = [s.forecast_features()], [s.active_cells()]
    for _ in range(steps):
        _, fb = s.integrate()
        if fb:
            break
        feats.append(s.forecast_features())
        snaps.append(s.active_cells())
    side = s.side_length
    s.close()
    xs, ys, ps = [], [], []
    for n in range(len(snaps) - horizon):
        xs.append(feats[n])
        ys.append(region_labels(snaps[n], snaps[n + horizon], side, max_err))
        ps.append(flagged(snaps[n], max_err))
    if not xs:
        raise RuntimeError("the run is shorter than the horizon")
    return RunData(np.concatenate(xs), np.concatenate(ys), np.concatenate(ps), len(snaps) - 1)


def scores(pred: np.ndarray, truth: np.ndarray) -> dict:
    tp = int((pred & truth).sum())
    fp = int((pred & ~truth).sum())
    fn = int((~pred & truth).sum())
    precision = tp / (tp + fp) if tp + fp else 0.0
    recall = tp / (tp + fn) if tp + fn else 0.0
    f1 = 2 * precision * recall / (precision + recall) if precision + recall else 0.0
    return {"precision": precision, "recall": recall, "f1": f1, "positives": int(pred.sum()), "tp": tp, "fp": fp,
            "fn": fn}


def best_threshold(prob: np.ndarray, truth: np.ndarray) -> float:
    """The probability cut with the highest F1 on (training) data."""
    best, cut = -1.0, 0.5
    for c in np.linspace(0.05, 0.95, 19):
        f = scores(prob >= c, truth)["f1"]
        if f > best:
            best, cut = f, float(c)
    return cut


def train_forecaster(runs: Sequence[RunData], n_in: int, epochs: int = 30, seed: int = 1, lr: float = 3e-3):
    """Trains a network on the runs; returns (network, probability cut, last-pass mean loss)."""
    x = np.concatenate([r.x for r in runs])
    y = np.concatenate([r.y for r in runs]).astype(np.float32)
    pw = float(min(max((y.size - y.sum()) / max(y.sum(), 1.0), 1.0), 20.0))
    net = Mlp(n_in, seed)
    loss = net.train(x, y, epochs=epochs, batch=512, lr=lr, pos_weight=pw, seed=seed + 1)
    cut = best_threshold(net.predict(x), y.astype(bool))
    return net, cut, loss


def run_with_forecast(solver: Solver, net: Mlp, cut: float, steps: int, interval: int = 8,
                      coarsen_every: int = 1) -> dict:
    """Advances `steps` global steps with the forecast-driven regrid: every `interval` steps the
    network marks the cells it expects the indicator to flag within its horizon (dg_set_hold: they are
    not coarsened until the next forecast), and coarsening runs every `coarsen_every` steps
    (dg_set_coarsen_interval; 1 = at every opportunity, as the reference). The plain indicator still
    splits what it flags at every substep, so a miss of the network costs a late split, never a
    missing one. With coarsening at every step only the held cells keep their level: the regrid stops
    coarsening cells that the indicator would flag again within the horizon (the split/unsplit churn
    behind a moving front) and leaves the rest of the grid to the plain rule.
    Returns the solver's split/unsplit counts, the cell updates and the number of held cells per
    forecast."""
    solver.set_coarsen_interval(coarsen_every)
    held = []
    fb = False
    for n in range(steps):
        if n % interval == 0:
            hold = net.predict(solver.forecast_features()) >= cut
            solver.set_hold(hold)
            held.append(int(hold.sum()))
        _, fb = solver.integrate()
        if fb:
            break
    st = solver.stats()
    return {"splits": st.n_splits, "unsplits": st.n_unsplits, "held": held, "force_break": fb,
            "cell_updates": st.cell_updates}
