"""Flat case files and cell snapshots.

A case file is the initial tree plus solver parameters in one little-endian binary blob
("DGCASE01"); it is what the drop-in host hands to the solver and what the CPU reference runner
reads, so both start from the same tree. A snapshot ("DGSNAP01") lists every active cell with its
tree level, time level, centre, time, conserved and primitive state.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from .models import ModelId, ModelShape
from .scene import RefineZone, Tree

N_PARAMS = 32
P = dict(
    SIDE=0, ACTIVE0=1, PERIODIC0=4, MAX_CFL=7, MAX_DT=8, MIN_ERR=9, MAX_ERR=10, MAX_LEVEL=11, MIN_LEVEL=12,
    GAMMA=13, NS_MU=14, NS_LAMBDA=15, GAMMA1=16, GAMMA2=17, P1=18, P2=19, CP1=20, CP2=21, CV1=22, CV2=23,
    MU1=24, MU2=25, LAMBDA1=26, LAMBDA2=27, SIGMA=28, PRUNED=29, POOL_CAP=30,
)


@dataclass
class SolverParams:
    """Config fields the integrator reads (integrator/integrator.hpp:80-86) and model constants.

    Multiphase defaults are the static initialisers of model/multi.hpp:50-62; note that
    cv1 = cp1 / 6.12 and cv2 = cp2 / 1.4 are evaluated once from the *default* gammas and are not
    updated when a case overrides gamma1/gamma2 (model/multi.hpp:57-58, :540-548).
    """

    side_length: float
    active_size: Sequence[float]
    periodic: Sequence[bool]
    max_cfl: float
    max_dt: float
    error_threshold: Sequence[float]  # (min_err, max_err)
    max_level: int
    min_level: int
    weights: Sequence[float]
    ns_mu: float = 0.0
    ns_lambda: float = 0.0
    gamma1: float = 6.12
    gamma2: float = 1.4
    P1: float = 343000000.0
    P2: float = 0.0
    cp1: float = 4181.0
    cp2: float = 1005.0
    cv1: float = 4181.0 / 6.12
    cv2: float = 1005.0 / 1.4
    mu1: float = 0.0
    mu2: float = 0.0
    lambda1: float = 0.0
    lambda2: float = 0.0
    sigma: float = 0.0
    zones: Sequence[RefineZone] = field(default_factory=list)
    limiter: int = 0  # dacti::integrator::slope id: minmod, unlimited, van_leer, superbee, von_alba_2, koren, first_order
    # GPU solver only (the reference runner ignores them): node slots left out of the upload by
    # prune_inactive, which still count towards the tree size, and a node-pool capacity (0: 1.5 x nodes)
    pruned_nodes: int = 0
    pool_capacity: int = 0

    def param_vector(self) -> np.ndarray:
        v = np.zeros(N_PARAMS, np.float64)
        v[P["SIDE"]] = self.side_length
        for d in range(3):
            v[P["ACTIVE0"] + d] = self.active_size[d] if d < len(self.active_size) else 0.0
            v[P["PERIODIC0"] + d] = 1.0 if d < len(self.periodic) and self.periodic[d] else 0.0
        v[P["MAX_CFL"]] = self.max_cfl
        v[P["MAX_DT"]] = self.max_dt
        v[P["MIN_ERR"]] = self.error_threshold[0]
        v[P["MAX_ERR"]] = self.error_threshold[1]
        v[P["MAX_LEVEL"]] = self.max_level
        v[P["MIN_LEVEL"]] = self.min_level
        v[P["GAMMA"]] = 1.4
        v[P["NS_MU"]] = self.ns_mu
        v[P["NS_LAMBDA"]] = self.ns_lambda
        for k in ("GAMMA1", "GAMMA2", "P1", "P2", "CP1", "CP2", "CV1", "CV2", "MU1", "MU2", "LAMBDA1", "LAMBDA2",
                  "SIGMA"):
            attr = {"GAMMA1": "gamma1", "GAMMA2": "gamma2"}.get(k, k if k in ("P1", "P2") else k.lower())
            v[P[k]] = getattr(self, attr)
        v[P["PRUNED"]] = float(self.pruned_nodes)
        v[P["POOL_CAP"]] = float(self.pool_capacity)
        return v


@dataclass
class Case:
    tree: Tree
    params: SolverParams

    @property
    def shape(self) -> ModelShape:
        return self.tree.shape


def prune_inactive(case: Case, pool_capacity: int = 0) -> Case:
    """The case without the nodes whose subtree holds no active leaf (the parts of the root box outside
    the active box, the inside of solid objects), for the GPU solver.

    Nothing the integrator computes reads those nodes: their faces towards active cells carry boundary
    conditions, subtree means skip inactive children, and a walk that meets a removed child (slot 0)
    treats it as the inactive leaf it stands for. Their number goes to ``pruned_nodes``, which the
    solver adds to its tree size wherever the reference's tree.size() enters (the garbage-collection
    trigger, impl/integrate.hpp:78-84), so results are unchanged. Node numbering changes, and the tree a
    writer reads back (dg_read_tree) lacks the removed nodes.
    """
    t = case.tree
    n = t.n_nodes
    keep = np.zeros(n, bool)
    keep[t.leaf_mask()] = True
    lv = t.level.astype(np.int64)
    order = np.argsort(-lv, kind="stable")
    # ancestors of active leaves, deepest level first
    for level in range(int(lv.max()), 0, -1):
        idx = order[lv[order] == level]
        par = t.parent[idx[keep[idx]]]
        keep[par] = True
    keep[0] = True
    if n > 1:
        keep[1] = True
    newidx = np.cumsum(keep).astype(np.int64) - 1
    newidx[~keep] = 0
    ch = t.children[keep]
    children = np.where(keep[ch], newidx[ch], 0).astype(np.int32)
    tree = Tree(t.shape, newidx[t.parent[keep]].astype(np.int32), children, t.level[keep].copy(),
                t.flags[keep].copy(), t.bc[keep].copy(), t.center[keep].copy(), t.p[keep].copy(), list(t.bcs))
    prm = dataclasses.replace(case.params, pruned_nodes=int(case.params.pruned_nodes + n - int(keep.sum())),
                              pool_capacity=int(pool_capacity))
    return Case(tree, prm)


def write_case(case: Case, path: str) -> None:
    t, prm = case.tree, case.params
    sh = t.shape
    E, D = sh.E, sh.dims
    with open(path, "wb") as f:
        f.write(b"DGCASE01")
        hdr = np.array([int(sh.model), D, t.n_nodes, len(t.bcs), len(prm.zones), int(prm.limiter), 0, 0], np.int32)
        f.write(hdr.tobytes())
        f.write(prm.param_vector().tobytes())
        f.write(np.asarray(prm.weights, np.float64).reshape(E).tobytes())
        for z in prm.zones:
            x0 = np.zeros(3)
            x1 = np.zeros(3)
            x0[: len(z.x0)] = z.x0
            x1[: len(z.x1)] = z.x1
            f.write(x0.tobytes() + x1.tobytes() + np.array([float(z.level)]).tobytes())
        for b in t.bcs:
            f.write(np.array([int(b.type), 0], np.int32).tobytes())
            f.write(np.asarray(b.p_in, np.float64).reshape(E).tobytes())
            f.write(np.asarray(b.normal, np.float64).reshape(D).tobytes())
            f.write(np.array([b.fade_in], np.float64).tobytes())
        f.write(t.parent.astype(np.int32).tobytes())
        f.write(t.children.astype(np.int32).tobytes())
        f.write(t.level.astype(np.int32).tobytes())
        f.write(t.flags.astype(np.uint32).tobytes())
        f.write(t.bc.astype(np.int32).tobytes())
        f.write(t.center.astype(np.float64).tobytes())
        f.write(t.p.astype(np.float64).tobytes())


@dataclass
class Snapshot:
    dims: int
    E: int
    step: int
    n_substeps: int
    tree_size: int
    n_in_clusters: int
    time: float
    global_dt: float
    updates: float
    tree_level: np.ndarray
    acti_level: np.ndarray
    center: np.ndarray
    t: np.ndarray
    u: np.ndarray
    p: np.ndarray
    error: np.ndarray
    max_dt: np.ndarray
    cfl: np.ndarray
    k: Optional[np.ndarray] = None  # model parameters (multi: mu, -, normal[D], kappa, smoothed alpha)

    @property
    def n(self) -> int:
        return int(self.tree_level.shape[0])

    def sorted(self, side_length: float) -> "Snapshot":
        """Cells ordered by (tree level, integer cell coordinates): a canonical order."""
        coords = cell_coords(self.center, self.tree_level, side_length)
        keys = [coords[:, d] for d in reversed(range(self.dims))] + [self.tree_level]
        o = np.lexsort(keys)
        return Snapshot(
            self.dims, self.E, self.step, self.n_substeps, self.tree_size, self.n_in_clusters, self.time,
            self.global_dt, self.updates, self.tree_level[o], self.acti_level[o], self.center[o], self.t[o],
            self.u[o], self.p[o], self.error[o], self.max_dt[o], self.cfl[o], None if self.k is None else self.k[o],
        )


def cell_coords(center: np.ndarray, level: np.ndarray, side_length: float) -> np.ndarray:
    """Integer cell index of each centre at its own tree level (root box centred at the origin)."""
    n_l = np.left_shift(np.int64(1), level.astype(np.int64))
    return np.floor((center / side_length + 0.5) * n_l[:, None]).astype(np.int64)


def read_snapshot(path: str) -> Snapshot:
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"DGSNAP01":
        raise ValueError("bad snapshot magic")
    hdr = np.frombuffer(buf, np.int32, 8, 8)
    D, E, n, n_in, step, nsub, tsz = (int(x) for x in hdr[:7])
    hd = np.frombuffer(buf, np.float64, 3, 40)
    base = D + 1 + 2 * E + 3
    n_par = ((len(buf) - 64) // max(n, 1) - 8) // 8 - base if n > 0 else 0
    rec = np.dtype([("lv", np.int32, 2), ("d", np.float64, base + n_par)])
    arr = np.frombuffer(buf, rec, n, 64)
    d = arr["d"]
    return Snapshot(
        D, E, step, nsub, tsz, n_in, float(hd[0]), float(hd[1]), float(hd[2]),
        arr["lv"][:, 0].copy(), arr["lv"][:, 1].copy(), d[:, :D].copy(), d[:, D].copy(),
        d[:, D + 1: D + 1 + E].copy(), d[:, D + 1 + E: D + 1 + 2 * E].copy(), d[:, D + 1 + 2 * E].copy(),
        d[:, D + 2 + 2 * E].copy(), d[:, D + 3 + 2 * E].copy(), d[:, base:].copy() if n_par > 0 else None,
    )


def read_case(path: str) -> Case:
    """Inverse of write_case."""
    from .models import BcType
    from .scene import BoundarySpec, RefineZone, Tree

    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"DGCASE01":
        raise ValueError("bad case magic")
    off = 8
    hdr = np.frombuffer(buf, np.int32, 8, off)
    off += 32
    model, D, n, nbc, nz, lim = (int(x) for x in hdr[:6])
    shape = ModelShape(ModelId(model), D)
    E, C, NF = shape.E, shape.C, shape.NF
    prm = np.frombuffer(buf, np.float64, N_PARAMS, off)
    off += 8 * N_PARAMS
    weights = np.frombuffer(buf, np.float64, E, off).copy()
    off += 8 * E
    zones = []
    for _ in range(nz):
        z = np.frombuffer(buf, np.float64, 7, off)
        off += 56
        zones.append(RefineZone(list(z[:3]), list(z[3:6]), int(z[6])))
    bcs = []
    for _ in range(nbc):
        tp = np.frombuffer(buf, np.int32, 2, off)
        off += 8
        pin = np.frombuffer(buf, np.float64, E, off).copy()
        off += 8 * E
        nrm = np.frombuffer(buf, np.float64, D, off).copy()
        off += 8 * D
        fade = float(np.frombuffer(buf, np.float64, 1, off)[0])
        off += 8
        bcs.append(BoundarySpec(BcType(int(tp[0])), list(pin), list(nrm), fade))

    def take(dtype, count, shape_=None):
        nonlocal off
        a = np.frombuffer(buf, dtype, count, off).copy()
        off += a.nbytes
        return a.reshape(shape_) if shape_ else a

    parent = take(np.int32, n)
    children = take(np.int32, n * C, (n, C))
    level = take(np.int32, n)
    flags = take(np.uint32, n)
    bc = take(np.int32, n * NF, (n, NF))
    center = take(np.float64, n * D, (n, D))
    p = take(np.float64, n * E, (n, E))
    tree = Tree(shape, parent, children, level, flags, bc, center, p, bcs)
    params = SolverParams(
        side_length=float(prm[P["SIDE"]]), active_size=[float(prm[P["ACTIVE0"] + d]) for d in range(D)],
        periodic=[bool(prm[P["PERIODIC0"] + d]) for d in range(D)], max_cfl=float(prm[P["MAX_CFL"]]),
        max_dt=float(prm[P["MAX_DT"]]), error_threshold=(float(prm[P["MIN_ERR"]]), float(prm[P["MAX_ERR"]])),
        max_level=int(prm[P["MAX_LEVEL"]]), min_level=int(prm[P["MIN_LEVEL"]]), weights=list(weights),
        ns_mu=float(prm[P["NS_MU"]]), ns_lambda=float(prm[P["NS_LAMBDA"]]), gamma1=float(prm[P["GAMMA1"]]),
        gamma2=float(prm[P["GAMMA2"]]), P1=float(prm[P["P1"]]), P2=float(prm[P["P2"]]), cp1=float(prm[P["CP1"]]),
        cp2=float(prm[P["CP2"]]), cv1=float(prm[P["CV1"]]), cv2=float(prm[P["CV2"]]), mu1=float(prm[P["MU1"]]),
        mu2=float(prm[P["MU2"]]), lambda1=float(prm[P["LAMBDA1"]]), lambda2=float(prm[P["LAMBDA2"]]),
        sigma=float(prm[P["SIGMA"]]), zones=zones, limiter=lim,
    )
    return Case(tree, params)
