"""One tree over two ranks on CPU (gloo): the Morton-range partition and the per-substep exchange of
dacti_b200/shard.py reproduce the one-rank face-flux sums bit for bit.

The fluxes are the reference's own arithmetic through the plain-C restatement (oracle/restate, the
test's checker). A rank starts with the records of its own leaves only (every other row NaN), gets the
records of the leaves across its boundary from the ghost exchange, evaluates the faces it owns, sends
the fluxes of faces whose other cell lives on the other rank back to that rank, and sums every cell's
faces in the same fixed order as the one-rank run."""
import ctypes
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT
from dacti_b200 import shard

LIB = os.path.join(ROOT, "oracle", "restate", "libdacti_restate.so")
W = 78  # doubles of one restated Cell record: size, t, centre[3], u, p, rhs, k, t_slope, slope[3], gradient[3]


def _tree():
    """Leaves of a 2D Euler quadtree on the unit square: the 16 x 16 base of the Lax-Liu case with the
    cells of a disc split once (hanging faces around it), seeded slopes and rhs."""
    from dacti_b200 import cases
    from dacti_b200.casefile import cell_coords
    case = cases.lax_liu3(base_level=4, levels=2)
    t = case.tree
    leaf = np.nonzero(t.leaf_mask())[0]
    lv0 = t.level[leaf].astype(np.int64)
    c0 = cell_coords(t.center[leaf], lv0, case.params.side_length)
    x0, p0 = t.center[leaf], t.p[leaf]
    split = np.hypot(x0[:, 0] - 0.1, x0[:, 1] + 0.05) < 0.25
    coords, lv, ctr, prim = [c0[~split]], [lv0[~split]], [x0[~split]], [p0[~split]]
    h = case.params.side_length * 0.5 ** lv0[split]
    for k in range(4):
        bits = np.array([k & 1, (k >> 1) & 1])
        coords.append(2 * c0[split] + bits)
        lv.append(lv0[split] + 1)
        ctr.append(x0[split] + (bits - 0.5) * 0.5 * h[:, None])
        prim.append(p0[split])
    coords, lv, ctr, prim = np.concatenate(coords), np.concatenate(lv), np.concatenate(ctr), np.concatenate(prim)
    rng = np.random.default_rng(7)
    rec = np.zeros((lv.size, W))
    rec[:, 0] = case.params.side_length * 0.5 ** lv
    rec[:, 2:4] = ctr
    rec[:, 12:16] = prim
    rec[:, 19:23] = 1e-3 * rng.standard_normal((lv.size, 4))       # rhs
    for d in range(2):
        rec[:, 39 + 7 * d:43 + 7 * d] = 0.1 * rng.standard_normal((lv.size, 4))  # slopes
    acti = rng.integers(0, 3, lv.size)
    return coords, lv, rec, acti


def _lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restate/libdacti_restate.so"], check=True,
                       capture_output=True)
    lb = ctypes.CDLL(LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    lb.ro_flux.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                           ctypes.c_int, dp]
    return lb


class RoModel(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("dims", ctypes.c_int)] + [
        (n, ctypes.c_double) for n in ("ns_mu", "ns_lambda", "gamma1", "gamma2", "P1", "P2", "cp1", "cp2", "cv1",
                                       "cv2", "mu1", "mu2", "lambda1", "lambda2", "sigma")]


def _model():
    return RoModel(0, 2)  # Euler 2D


def _face_flux(lb, m, rec, owner, other, dim, dr):
    """Model::flux of the face of `owner` in direction dr towards `other` (impl/flux.hpp:32-39): the
    owner is the left state for dr = 1 and the right state for dr = 0; the face sits on the owner's side."""
    dp = ctypes.POINTER(ctypes.c_double)
    left, right = (owner, other) if dr == 1 else (other, owner)
    cl = np.ascontiguousarray(rec[left])
    cr = np.ascontiguousarray(rec[right])
    fc = np.zeros(3)
    fc[:2] = rec[owner, 2:4]
    fc[dim] += rec[owner, 0] * (dr - 0.5)
    F = np.zeros(4)
    lb.ro_flux(ctypes.byref(m), cl.ctypes.data_as(dp), cr.ctypes.data_as(dp), fc.ctypes.data_as(dp),
               float(rec[owner, 0]), 0.0, 1e-3, dim, F.ctypes.data_as(dp))
    return F


def _sums(lb, m, rec, level, faces, mine, returned, remote=frozenset()):
    """Fixed-order flux sum of every cell in `mine`: faces 2 dim + dir in order, the fine fluxes of a
    hanging face in child order. A face owned by a leaf of another rank (in `remote`) takes its flux
    from `returned` (keyed by (owner, dim, owner's dir, cell)); all other faces are evaluated here."""
    out = {}
    for i in mine:
        s = np.zeros(4)
        for f in sorted(faces[i], key=lambda f: 2 * f.dim + f.dir):
            term = np.zeros(4)
            for j in f.others:
                if shard.owns(level, i, j, f.dir):
                    F = _face_flux(lb, m, rec, i, j, f.dim, f.dir)
                    term = term + (-F if f.dir == 1 else F)
                else:
                    key = (j, f.dim, 1 - f.dir, i)
                    F = returned[key] if j in remote else _face_flux(lb, m, rec, j, i, f.dim, 1 - f.dir)
                    term = term + (-F if f.dir == 1 else F)
            s = s + term
        out[i] = s
    return out


def _free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        coords, lv, full, acti = _tree()
        keys = shard.morton_keys(coords, lv, int(lv.max()))
        rank_of = shard.partition(keys, 2.0 ** acti, world)
        faces = shard.face_neighbours(coords, lv, 2, (1, 1))
        plan = shard.build_plans(rank_of, faces, lv, world)[rank]
        mine = np.nonzero(rank_of == rank)[0]
        rec = np.full_like(full, np.nan)
        rec[mine] = full[mine]
        for s, rows in shard.exchange_ghosts(plan, rec).items():
            rec[plan.ghosts_from[s]] = rows
        lb, m = _lib(), _model()
        # faces this rank owns towards a cell of another rank, evaluated here and sent there
        fl = {s: np.array([_face_flux(lb, m, rec, o, j, d, dr) for (o, d, dr, j) in lst]).reshape(-1, 4)
              for s, lst in plan.returns_to.items()}
        got = shard.exchange_returns(plan, fl, 4)
        returned = {}
        for s, rows in got.items():
            for key, row in zip(plan.returns_from[s], rows):
                returned[key] = row
        remote = frozenset(int(x) for x in np.nonzero(rank_of != rank)[0])
        sums = _sums(lb, m, rec, lv, faces, mine, returned, remote)
        q.put((rank, {int(k): v.tobytes() for k, v in sums.items()},
               {s: int(v.size) for s, v in plan.ghosts_from.items()}, len(returned)))
    finally:
        dist.destroy_process_group()


def test_partition_is_contiguous_and_balanced():
    coords, lv, _, acti = _tree()
    keys = shard.morton_keys(coords, lv, int(lv.max()))
    w = 2.0 ** acti
    for world in (2, 3, 4):
        r = shard.partition(keys, w, world)
        order = np.argsort(keys)
        assert np.all(np.diff(r[order]) >= 0)  # contiguous Morton ranges
        loads = np.bincount(r, weights=w, minlength=world)
        assert loads.max() - loads.min() <= 2 * w.max()


def test_two_ranks_reproduce_one_rank_flux_sums_bitwise():
    coords, lv, rec, acti = _tree()
    faces = shard.face_neighbours(coords, lv, 2, (1, 1))
    assert any(f.finer for fl in faces for f in fl)  # hanging faces are part of the case
    lb, m = _lib(), _model()
    ref = _sums(lb, m, rec, lv, faces, range(len(lv)), {})
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    got = {}
    for _, sums, ghosts, _ in res:
        assert sum(ghosts.values()) > 0  # each rank needed records from the other
        got.update(sums)
    assert sum(r[3] for r in res) > 0  # fluxes of faces owned across the boundary went back
    assert sorted(got) == list(range(len(lv)))
    for i, v in ref.items():
        assert got[i] == v.tobytes(), i
