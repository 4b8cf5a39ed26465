"""One tree on several GPUs, one rank per GPU: the partition of the active leaves and the exchange of
one level substep.

Partition. The active leaves are ordered along the Z-order (Morton) curve of their cells and cut
into contiguous ranges of equal weight, a leaf weighing 2^acti_level: the number of times a global
step updates it (impl/integrate.hpp:26-67 runs level L 2^L times). A Morton range is a compact region
of the domain, so a rank's surface, and with it the exchanged data, stays small.

Exchange of a level substep, the coupling across rank boundaries of flux_update
(impl/flux.hpp:11-97):
- ghost states: every rank receives the reconstruction records (primitive state, Hancock rhs,
  slopes, curvature and normal, centre, size, time) of the other ranks' leaves that touch its own;
- flux return: every face carries one flux, evaluated by the rank of its owner (the finer cell; at
  equal levels the cell on the left, impl/flux.hpp:58-59). When the other cell of the face lives on
  another rank, the owner's rank sends the face's flux there, and that rank adds it into the cell in
  the cell's own fixed face order, as on one rank: the coarse side of a fine-coarse face collects its
  fine fluxes this way (impl/flux.hpp:80-91).
Both transfers are point to point between ranks that share a boundary (torch.distributed send/recv:
NCCL over NVLink between GPUs, gloo between CPU processes), no collective.

With local time stepping the plans are per ACTI level (build_lts_plans): in the substep of level L only
the faces owned by level-L leaves carry a flux, under the reference's ownership rule with ACTI levels
(owns_lts), and a slower leaf across the boundary collects the returned fluxes over several substeps
before its own update.

This module is the host side of that design: the partition, the plan of which leaves and faces cross
which rank boundary, and the packing and unpacking of the transfers. The device kernels of the solver
do not read ghost buffers yet; one tree runs on one GPU.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, List, Sequence, Tuple

import numpy as np


def morton_keys(coords: np.ndarray, level: np.ndarray, max_level: int) -> np.ndarray:
    """Z-order keys of cells given by integer coordinates at their own level: each cell's coordinates
    are scaled to `max_level` and their bits interleaved (dimension 0 lowest)."""
    coords = np.asarray(coords, np.int64)
    level = np.asarray(level, np.int64)
    n, dims = coords.shape
    scaled = coords << (max_level - level)[:, None]
    keys = np.zeros(n, np.uint64)
    for b in range(max_level):
        for d in range(dims):
            bit = ((scaled[:, d] >> b) & 1).astype(np.uint64)
            keys |= bit << np.uint64(b * dims + d)
    return keys


def partition(keys: np.ndarray, weights: np.ndarray, world: int) -> np.ndarray:
    """Rank of every leaf: contiguous ranges of the Morton order holding (as nearly as whole leaves
    allow) 1/world of the total weight each."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.argsort(keys, kind="stable")
    w = np.asarray(weights, np.float64)[order]
    cum = np.cumsum(w) - 0.5 * w  # weight before each leaf's midpoint
    total = float(w.sum())
    r_sorted = np.minimum((cum * world / max(total, 1e-300)).astype(np.int64), world - 1)
    rank = np.empty(len(keys), np.int64)
    rank[order] = r_sorted
    return rank


@dataclass
class Face:
    """One flux-carrying face seen from `cell`: its neighbours across face (dim, dir). `others` holds
    one leaf (same level or coarser) or the finer leaves touching the face, in child order."""
    cell: int
    dim: int
    dir: int
    others: Tuple[int, ...]
    finer: bool


def face_neighbours(coords: np.ndarray, level: np.ndarray, dims: int, n_root: Sequence[int]) -> List[List[Face]]:
    """Face neighbours of every leaf of a 2:1-balanced set of leaves covering a box of n_root[d] << l
    cells per dimension at level l. Faces on the box's boundary have no neighbour (a boundary
    condition) and are left out."""
    coords = np.asarray(coords, np.int64)
    level = np.asarray(level, np.int64)
    index: Dict[tuple, int] = {(int(level[i]), *map(int, coords[i])): i for i in range(len(level))}
    out: List[List[Face]] = []
    for i in range(len(level)):
        faces: List[Face] = []
        li = int(level[i])
        for dim in range(dims):
            for dr in (0, 1):
                c = list(map(int, coords[i]))
                c[dim] += 1 if dr else -1
                if c[dim] < 0 or c[dim] >= (int(n_root[dim]) << li):
                    continue
                j = index.get((li, *c))
                if j is not None:
                    faces.append(Face(i, dim, dr, (j,), False))
                    continue
                parent = (li - 1, *[x >> 1 for x in c])
                if parent in index:
                    faces.append(Face(i, dim, dr, (index[parent],), False))
                    continue
                # finer: the children of the same-level cell that touch the face, in child order
                fine = []
                for k in range(1 << dims):
                    if ((k >> dim) & 1) != (1 - dr):
                        continue
                    cc = tuple(2 * c[d] + ((k >> d) & 1) for d in range(dims))
                    jj = index.get((li + 1, *cc))
                    if jj is None:
                        raise ValueError("leaves are not 2:1 balanced")
                    fine.append(jj)
                faces.append(Face(i, dim, dr, tuple(fine), True))
        out.append(faces)
    return out


def owns(level: np.ndarray, i: int, j: int, dir_i: int) -> bool:
    """Whether leaf i owns its face towards leaf j in direction dir_i (impl/flux.hpp:58-59 with a single
    time level): the finer cell, at equal levels the cell on the left (the face is its + face)."""
    return bool(level[i] > level[j] or (level[i] == level[j] and dir_i == 1))


@dataclass
class Plan:
    """Who needs what across rank boundaries, for one rank.

    ghosts_from[s]: leaves of rank s whose records this rank needs (sorted);
    ghosts_to[s]:   this rank's leaves that rank s needs (sorted);
    returns_to[s]:  (face-owner leaf, dim, dir, receiving leaf of rank s) of the faces this rank
                    evaluates for a cell of rank s, in a fixed order;
    returns_from[s]: the same list as rank s builds it for this rank.
    """
    rank: int
    ghosts_from: Dict[int, np.ndarray]
    ghosts_to: Dict[int, np.ndarray]
    returns_to: Dict[int, List[Tuple[int, int, int, int]]]
    returns_from: Dict[int, List[Tuple[int, int, int, int]]]


def build_plans(rank_of: np.ndarray, faces: List[List[Face]], level: np.ndarray, world: int) -> List[Plan]:
    """The exchange plan of every rank; every rank can build all of them from the same inputs, so
    the plans need no communication."""
    need = [[set() for _ in range(world)] for _ in range(world)]
    ret: List[List[List[Tuple[int, int, int, int]]]] = [[[] for _ in range(world)] for _ in range(world)]
    for fl in faces:
        for f in fl:
            r = int(rank_of[f.cell])
            for j in f.others:
                s = int(rank_of[j])
                if s != r:
                    need[r][s].add(j)
                    # the owner's rank evaluates the face; a remote non-owner gets the flux back
                    if owns(level, f.cell, j, f.dir):
                        ret[r][s].append((f.cell, f.dim, f.dir, j))
    plans = []
    for r in range(world):
        plans.append(Plan(
            r,
            {s: np.array(sorted(need[r][s]), np.int64) for s in range(world) if s != r},
            {s: np.array(sorted(need[s][r]), np.int64) for s in range(world) if s != r},
            {s: sorted(ret[r][s]) for s in range(world) if s != r},
            {s: sorted(ret[s][r]) for s in range(world) if s != r},
        ))
    return plans


def _exchange(sends: Dict[int, np.ndarray], recv_shapes: Dict[int, tuple], dtype) -> Dict[int, np.ndarray]:
    """Point-to-point transfer of one array per peer (torch.distributed isend/irecv), no collective."""
    import torch
    import torch.distributed as dist
    reqs, bufs = [], {}
    for s, shape in recv_shapes.items():
        bufs[s] = torch.empty(shape, dtype=dtype)
        reqs.append(dist.irecv(bufs[s], src=s))
    for s, arr in sends.items():
        reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(arr)), dst=s))
    for q in reqs:
        q.wait()
    return {s: b.numpy() for s, b in bufs.items()}


def exchange_ghosts(plan: Plan, records: np.ndarray) -> Dict[int, np.ndarray]:
    """Ghost records: `records` holds one row per leaf (only this rank's rows are read); returns, per
    peer, the rows of plan.ghosts_from[peer] in that order."""
    import torch
    sends = {s: records[idx] for s, idx in plan.ghosts_to.items() if idx.size}
    shapes = {s: (idx.size, records.shape[1]) for s, idx in plan.ghosts_from.items() if idx.size}
    return _exchange(sends, shapes, torch.float64)


def exchange_returns(plan: Plan, fluxes: Dict[int, np.ndarray], width: int) -> Dict[int, np.ndarray]:
    """Flux return: fluxes[peer] holds one row per entry of plan.returns_to[peer]; returns, per peer,
    the rows of plan.returns_from[peer]."""
    import torch
    sends = {s: fluxes[s] for s, lst in plan.returns_to.items() if lst}
    shapes = {s: (len(lst), width) for s, lst in plan.returns_from.items() if lst}
    return _exchange(sends, shapes, torch.float64)


# ------------------------------------------------------------------------------------------------
# Local time stepping across rank boundaries. With ACTI levels a face is evaluated in the substeps of
# its owner's level, and the owner is not always the finer or left cell: impl/flux.hpp:52-59 lets cell
# i evaluate its face towards leaf j when j is not faster (acti_j <= acti_i) and j is coarser, or at the
# same tree level the face is i's + face or j is slower. A slower cell therefore collects the fluxes
# of its faster neighbours over several of their substeps before its own update; across a rank
# boundary those fluxes come back to its rank substep by substep and go into its accumulator in the
# cell's fixed face order, as on one rank. The exchange plans are per ACTI level: at the substep of
# level L only the faces owned by level-L cells carry a flux, so only their other cells' records are
# fetched and only their fluxes are returned.
# ------------------------------------------------------------------------------------------------

def owns_lts(level: np.ndarray, acti: np.ndarray, i: int, j: int, dir_i: int) -> bool:
    """Whether leaf i evaluates the flux of its face (direction dir_i) towards leaf j in its own
    substeps (impl/flux.hpp:52-59). A finer j is never owned from the coarse side."""
    li, lj, ai, aj = int(level[i]), int(level[j]), int(acti[i]), int(acti[j])
    return aj <= ai and (lj < li or (lj == li and (dir_i == 1 or aj < ai)))


def face_owner_lts(level: np.ndarray, acti: np.ndarray, f: Face, k: int):
    """(owner, other, dim, owner's direction) of the flux between f.cell and its neighbour k across
    face f, or None when neither side evaluates it (a quirk of the rule: a coarse cell faster than
    its finer neighbours leaves their common face without a flux, as the reference does)."""
    i = f.cell
    if owns_lts(level, acti, i, k, f.dir):
        return (i, k, f.dim, f.dir)
    if owns_lts(level, acti, k, i, 1 - f.dir):
        return (k, i, f.dim, 1 - f.dir)
    return None


def build_lts_plans(rank_of: np.ndarray, faces: List[List[Face]], level: np.ndarray, acti: np.ndarray,
                    world: int) -> List[Dict[int, Plan]]:
    """Per rank, per ACTI level L: the Plan of the substep of level L. ghosts_from[s] lists the leaves
    of rank s that are the other cell of a face owned by one of this rank's level-L leaves;
    returns_to[s] lists (owner, dim, owner's dir, receiving leaf) of those faces whose other cell is
    on rank s. Every rank builds all plans from the same inputs."""
    levels = sorted(set(int(a) for a in acti))
    need = {L: [[set() for _ in range(world)] for _ in range(world)] for L in levels}
    ret = {L: [[[] for _ in range(world)] for _ in range(world)] for L in levels}
    for fl in faces:
        for f in fl:
            for k in f.others:
                o = face_owner_lts(level, acti, f, k)
                if o is None or o[0] != f.cell:
                    continue  # each evaluated face once, from its owner's face list
                owner, other, dim, d = o
                L = int(acti[owner])
                r, s = int(rank_of[owner]), int(rank_of[other])
                if r != s:
                    need[L][r][s].add(other)
                    ret[L][r][s].append((owner, dim, d, other))
    plans: List[Dict[int, Plan]] = []
    for r in range(world):
        per: Dict[int, Plan] = {}
        for L in levels:
            per[L] = Plan(
                r,
                {s: np.array(sorted(need[L][r][s]), np.int64) for s in range(world) if s != r},
                {s: np.array(sorted(need[L][s][r]), np.int64) for s in range(world) if s != r},
                {s: sorted(ret[L][r][s]) for s in range(world) if s != r},
                {s: sorted(ret[L][s][r]) for s in range(world) if s != r},
            )
        plans.append(per)
    return plans


def lts_schedule(max_level: int) -> List[int]:
    """ACTI levels of the substeps of one global step in the order impl/integrate.hpp:26-67 runs them:
    the sequence counter steps through 1 .. 2^max_level, and at each value every level L whose period
    2^(max_level - L) divides it runs, finest first."""
    out = []
    for seq in range(1, (1 << max_level) + 1):
        for L in range(max_level, -1, -1):
            if seq % (1 << (max_level - L)) == 0:
                out.append(L)
    return out


# ------------------------------------------------------------------------------------------------
# Reductions over ranks. The step itself needs none (global_dt is fixed at construction); the
# construction and the diagnostics do.
# ------------------------------------------------------------------------------------------------

def initial_global_dt(local_max_dt: float, max_dt_cfg: float) -> float:
    """integrator/integrator.hpp:100-150 over ranks: the largest max_delta_time of any active leaf (a MAX
    all-reduce, exact in any order), then min(0.9 x that, the configured max_dt)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local_max_dt)], dtype=torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return min(0.9 * float(t[0]), float(max_dt_cfg))


def rank_ordered_sum(local: np.ndarray) -> np.ndarray:
    """Sum over ranks of per-rank partial sums (conservation totals, regrid counts): the parts are
    gathered and added in rank order on every rank, so every rank and every run gets the same bits,
    which an all-reduce in an order of the library's choosing does not promise."""
    import torch
    import torch.distributed as dist
    x = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64))
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x.numpy().copy()
    parts = [torch.empty_like(x) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, x)
    s = np.zeros_like(local, dtype=np.float64)
    for p in parts:
        s = s + p.numpy()
    return s
