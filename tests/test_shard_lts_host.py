"""One global step of local time stepping on one tree split over two ranks (gloo, CPU): the per-level
exchange plans of dacti_b200/shard.py reproduce the one-rank step bit for bit.

The step is the flux coupling of the LTS schedule (impl/integrate.hpp:26-67 with impl/flux.hpp:11-97):
substeps in the reference's level order; in the substep of level L every face owned by a level-L
leaf is evaluated once with the owner's time and size, every leaf adds its fixed-order sum of those
fluxes into its accumulator, and the level-L leaves are updated (u += accumulator / volume, primitive
state, t += dt_L) and reset their accumulator. Slower leaves thus collect fluxes over several faster
substeps before their own update, across the rank boundary too. Fluxes and the primitive recovery are
the reference's arithmetic through the plain-C restatement (the test's checker). Slopes and rhs keep
their seeded values; the ACTI reassignment and the regrid are not part of this step."""
import ctypes
import os
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT
from dacti_b200 import shard
from test_shard_host import _free_port, _lib, _model, _tree

GLOBAL_DT = 2e-4


def _with_prim_cons(lb):
    dp = ctypes.POINTER(ctypes.c_double)
    lb.ro_prim_from_cons.argtypes = [ctypes.c_void_p, dp, dp]
    lb.ro_cons_from_prim.argtypes = [ctypes.c_void_p, dp, dp]
    lb.ro_max_delta_time.argtypes = [ctypes.c_void_p, dp]
    lb.ro_max_delta_time.restype = ctypes.c_double
    return lb


MAX_DT_CFG = 1.0


def _local_max_dt(lb, m, rec, cells):
    """The largest Model::max_delta_time over `cells` (integrator/integrator.hpp:113-114)."""
    dp = ctypes.POINTER(ctypes.c_double)
    g = -np.inf
    for j in cells:
        row = np.ascontiguousarray(rec[j])
        g = max(g, lb.ro_max_delta_time(ctypes.byref(m), row.ctypes.data_as(dp)))
    return g


def _totals(rec, cells):
    """Conserved totals sum(u volume) over `cells` in ascending order."""
    s = np.zeros(4)
    for j in sorted(cells):
        s = s + rec[j, 5:9] * (rec[j, 0] * rec[j, 0])
    return s


def _start(lb, m):
    """The seeded tree with conserved states from its primitive ones, ACTI levels 0..2, t = 0."""
    coords, lv, rec, acti = _tree()
    dp = ctypes.POINTER(ctypes.c_double)
    for i in range(lv.size):
        p = np.ascontiguousarray(rec[i, 12:16])
        u = np.zeros(4)
        lb.ro_cons_from_prim(ctypes.byref(m), p.ctypes.data_as(dp), u.ctypes.data_as(dp))
        rec[i, 5:9] = u
    return coords, lv, rec, acti


def _flux(lb, m, rec, owner, other, dim, dr, dtL):
    """Model::flux of the owner's face (impl/flux.hpp:25-32): the owner's size and time, t1 = t0 + dt_L;
    the owner is the left state for dr = 1 and the right state for dr = 0."""
    dp = ctypes.POINTER(ctypes.c_double)
    left, right = (owner, other) if dr == 1 else (other, owner)
    cl = np.ascontiguousarray(rec[left])
    cr = np.ascontiguousarray(rec[right])
    fc = np.zeros(3)
    fc[:2] = rec[owner, 2:4]
    fc[dim] += rec[owner, 0] * (dr - 0.5)
    t0 = float(rec[owner, 1])
    F = np.zeros(4)
    lb.ro_flux(ctypes.byref(m), cl.ctypes.data_as(dp), cr.ctypes.data_as(dp), fc.ctypes.data_as(dp),
               float(rec[owner, 0]), t0, t0 + dtL, dim, F.ctypes.data_as(dp))
    return F


def _terms(lv, acti, faces, cells, L, flux_of):
    """Each cell's sum of the fluxes of the level-L substep: faces 2 dim + dir in order, the fine
    fluxes of a hanging face in child order, signed as the reference adds them (impl/flux.hpp:80-91)."""
    out = {}
    for j in cells:
        s = np.zeros(4)
        for f in sorted(faces[j], key=lambda f: 2 * f.dim + f.dir):
            term = np.zeros(4)
            for k in f.others:
                o = shard.face_owner_lts(lv, acti, f, k)
                if o is None or int(acti[o[0]]) != L:
                    continue
                F = flux_of(o, j)
                term = term + (-F if f.dir == 1 else F)
            s = s + term
        out[j] = s
    return out


def _update(lb, m, rec, acc, cells, dtL):
    dp = ctypes.POINTER(ctypes.c_double)
    for j in cells:
        u = rec[j, 5:9] + acc[j] / (rec[j, 0] * rec[j, 0])
        p = np.zeros(4)
        uc = np.ascontiguousarray(u)
        lb.ro_prim_from_cons(ctypes.byref(m), uc.ctypes.data_as(dp), p.ctypes.data_as(dp))
        rec[j, 5:9] = u
        rec[j, 12:16] = p
        rec[j, 1] = rec[j, 1] + dtL
        acc[j] = np.zeros(4)


def _one_rank(lb, m, coords, lv, rec, acti, faces):
    acc = {j: np.zeros(4) for j in range(lv.size)}
    Lmax = int(acti.max())
    for L in shard.lts_schedule(Lmax):
        dtL = GLOBAL_DT / (1 << L)
        cache = {}

        def flux_of(o, j):
            if o not in cache:
                cache[o] = _flux(lb, m, rec, o[0], o[1], o[2], o[3], dtL)
            return cache[o]

        terms = _terms(lv, acti, faces, range(lv.size), L, flux_of)
        for j in range(lv.size):
            acc[j] = acc[j] + terms[j]
        _update(lb, m, rec, acc, [j for j in range(lv.size) if acti[j] == L], dtL)
    return rec


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lb, m = _with_prim_cons(_lib()), _model()
        coords, lv, full, acti = _start(lb, m)
        keys = shard.morton_keys(coords, lv, int(lv.max()))
        rank_of = shard.partition(keys, 2.0 ** acti, world)
        faces = shard.face_neighbours(coords, lv, 2, (1, 1))
        plans = shard.build_lts_plans(rank_of, faces, lv, acti, world)[rank]
        mine = [int(j) for j in np.nonzero(rank_of == rank)[0]]
        mine_set = set(mine)
        rec = np.full_like(full, np.nan)
        rec[mine] = full[mine]
        gdt = shard.initial_global_dt(_local_max_dt(lb, m, rec, mine), MAX_DT_CFG)
        acc = {j: np.zeros(4) for j in mine}
        returned_total, slower_receivers = 0, 0
        for L in shard.lts_schedule(int(acti.max())):
            plan = plans[L]
            dtL = GLOBAL_DT / (1 << L)
            # the records of the other cells of this rank's level-L faces, as their ranks hold them now
            for s, rows in shard.exchange_ghosts(plan, rec).items():
                rec[plan.ghosts_from[s]] = rows
            cache = {}
            for i in mine:
                if acti[i] != L:
                    continue
                for f in faces[i]:
                    for k in f.others:
                        o = shard.face_owner_lts(lv, acti, f, k)
                        if o is not None and o[0] == i:
                            cache[o] = _flux(lb, m, rec, o[0], o[1], o[2], o[3], dtL)
            sends = {s: np.array([cache[(o, r, d, dr)] for (o, d, dr, r) in lst]).reshape(-1, 4)
                     for s, lst in plan.returns_to.items()}
            returned = {}
            for s, rows in shard.exchange_returns(plan, sends, 4).items():
                for key, row in zip(plan.returns_from[s], rows):
                    returned[key] = row
                    returned_total += 1
                    slower_receivers += int(acti[key[3]] < L)

            def flux_of(o, j):
                if o[0] in mine_set:
                    return cache[o]
                return returned[(o[0], o[2], o[3], j)]

            terms = _terms(lv, acti, faces, mine, L, flux_of)
            for j in mine:
                acc[j] = acc[j] + terms[j]
            _update(lb, m, rec, acc, [j for j in mine if acti[j] == L], dtL)
        totals = shard.rank_ordered_sum(_totals(rec, mine))
        q.put((rank, {j: rec[j].tobytes() for j in mine}, returned_total, slower_receivers, gdt, totals.tobytes()))
    finally:
        dist.destroy_process_group()


def test_lts_plans_cover_every_owned_face_once():
    _, lv, _, acti = _tree()
    coords = _tree()[0]
    faces = shard.face_neighbours(coords, lv, 2, (1, 1))
    seen = set()
    for fl in faces:
        for f in fl:
            for k in f.others:
                o = shard.face_owner_lts(lv, acti, f, k)
                if o is not None:
                    # the same owner, other and direction from both sides of the face
                    seen.add(o)
    for (owner, other, dim, d) in seen:
        assert shard.owns_lts(lv, acti, owner, other, d)
        assert not shard.owns_lts(lv, acti, other, owner, 1 - d)
    assert len({int(acti[o[0]]) for o in seen}) == 3  # faces evaluated in substeps of all three levels
    assert shard.lts_schedule(2) == [2, 2, 1, 2, 2, 1, 0]


def test_two_ranks_reproduce_one_rank_lts_step_bitwise():
    lb, m = _with_prim_cons(_lib()), _model()
    coords, lv, rec, acti = _start(lb, m)
    faces = shard.face_neighbours(coords, lv, 2, (1, 1))
    ref = _one_rank(lb, m, coords, lv, rec.copy(), acti, faces)
    assert np.isfinite(_local_max_dt(lb, m, rec, range(lv.size)))
    assert np.allclose(ref[:, 1], GLOBAL_DT, rtol=1e-12, atol=0.0)  # every leaf reached the step's end
    assert np.isfinite(ref[:, 5:9]).all() and not np.array_equal(ref[:, 5:9], rec[:, 5:9])
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    # the reductions: the initial global dt over ranks equals one rank's; the totals are the per-rank
    # sums added in rank order, the same bits on both ranks
    keys = shard.morton_keys(coords, lv, int(lv.max()))
    rank_of = shard.partition(keys, 2.0 ** acti, 2)
    one_dt = min(0.9 * _local_max_dt(lb, m, rec, range(lv.size)), MAX_DT_CFG)
    assert all(r[4] == one_dt for r in res)
    parts = [_totals(ref, [j for j in range(lv.size) if rank_of[j] == r]) for r in range(2)]
    want = np.zeros(4)
    for p in parts:
        want = want + p
    assert all(r[5] == want.tobytes() for r in res)
    assert np.allclose(want, _totals(ref, range(lv.size)), rtol=1e-12, atol=0.0)
    got = {}
    for r in res:
        got.update(r[1])
    assert sorted(got) == list(range(lv.size))
    assert sum(r[2] for r in res) > 0  # fluxes crossed the rank boundary
    assert sum(r[3] for r in res) > 0  # some went to slower cells, to be summed over several substeps
    for j in range(lv.size):
        assert got[j] == ref[j].tobytes(), j
