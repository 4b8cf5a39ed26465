"""The plain-C restatement (oracle/restate) reproduces the reference's model arithmetic bit for bit.

Known-answer vectors under tests/golden/kat were produced by DACTI's own headers
(oracle/ref/kat.cpp via oracle/_ref/dacti_ref_kat) for seeded random inputs. File layout: int32
header {magic, model, dims, n_flux, n_bflux, n_cell, n_lim, n_est}, 17 model constants, then the
records (doubles):
  flux:  cell cn (78), cell cp (78), face centre[3], side, t0, t1, dim, F[11]
  bflux: cell (78), type, p_in[7], normal[3], fade_in, side, t0, t1, dim, dir, F[11]
  cell:  cell (78), du[11], prim(u)[7], cons(p)[7], max_dt, rhs[7], source[7], grad_input[6]
  lim:   s1, s2, minmod, unlimited, van_leer, superbee, von_alba_2, koren, first_order
  est:   cell (78), weights[7], neighbour states[6][7], present[6], estimate
A cell is {size, t, center[3], u[7], p[7], rhs[7], k[7], t_slope[6], slope[3][7], gradient[3][6]}.
"""
import ctypes
import glob
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

LIB = os.path.join(ROOT, "oracle", "restate", "libdacti_restate.so")
KATS = sorted(glob.glob(os.path.join(GOLDEN, "kat", "kat_*.bin")))


class RoModel(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("dims", ctypes.c_int)] + [
        (n, ctypes.c_double) for n in ("ns_mu", "ns_lambda", "gamma1", "gamma2", "P1", "P2", "cp1", "cp2", "cv1",
                                       "cv2", "mu1", "mu2", "lambda1", "lambda2", "sigma")]


class RoCell(ctypes.Structure):
    _fields_ = [("data", ctypes.c_double * 78)]


class RoBc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("p_in", ctypes.c_double * 7), ("normal", ctypes.c_double * 3),
                ("fade_in", ctypes.c_double)]


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restate/libdacti_restate.so"], check=True,
                       capture_output=True)
    lb = ctypes.CDLL(LIB)
    P = ctypes.POINTER
    dp = P(ctypes.c_double)
    lb.ro_flux.argtypes = [P(RoModel), P(RoCell), P(RoCell), dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                           ctypes.c_int, dp]
    lb.ro_boundary_flux.argtypes = [P(RoModel), P(RoBc), P(RoCell), ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int, dp]
    lb.ro_prim_from_cons.argtypes = [P(RoModel), dp, dp]
    lb.ro_cons_from_prim.argtypes = [P(RoModel), dp, dp]
    lb.ro_max_delta_time.argtypes = [P(RoModel), P(RoCell)]
    lb.ro_max_delta_time.restype = ctypes.c_double
    lb.ro_compute_rhs.argtypes = [P(RoModel), P(RoCell)]
    lb.ro_source.argtypes = [P(RoModel), P(RoCell), dp, dp]
    lb.ro_grad_input.argtypes = [P(RoModel), dp, dp]
    lb.ro_limit.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
    lb.ro_limit.restype = ctypes.c_double
    lb.ro_estimate.argtypes = [P(RoModel), dp, P(RoCell), dp, P(ctypes.c_int)]
    lb.ro_estimate.restype = ctypes.c_double
    return lb


def _arr(x):
    a = np.ascontiguousarray(x, np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _cell(v):
    c = RoCell()
    c.data[:] = list(v)
    return c


def _load(path):
    buf = open(path, "rb").read()
    hdr = np.frombuffer(buf, np.int32, 8, 0)
    magic, model, dims, nf, nb, nc, nl, ne = (int(x) for x in hdr)
    assert magic == 0x3154414B
    d = np.frombuffer(buf, np.float64, offset=32)
    consts, d = d[:17], d[17:]
    m = RoModel(model, dims, *consts[:15])
    recs = {}
    for name, n, w in (("flux", nf, 174), ("bflux", nb, 106), ("cell", nc, 124), ("lim", nl, 9), ("est", ne, 134)):
        recs[name] = d[: n * w].reshape(n, w)
        d = d[n * w:]
    assert d.size == 0
    return m, recs


@pytest.mark.parametrize("path", KATS, ids=[os.path.basename(p) for p in KATS])
def test_kat_vectors_are_mostly_physical(path):
    _, r = _load(path)
    assert np.isfinite(r["flux"][:, 163:]).mean() > 0.95 and np.isfinite(r["bflux"][:, 95:]).mean() > 0.95


@pytest.mark.parametrize("path", KATS, ids=[os.path.basename(p) for p in KATS])
def test_restatement_matches_reference_bitwise(lib, path):
    m, r = _load(path)
    E = m.dims + (4 if m.model == 2 else 2)
    NFL = E + (m.dims + 1 if m.model == 2 else 0)
    G = m.dims + 3 if m.model == 2 else (m.dims + 1 if m.model == 1 else 0)
    F = np.zeros(11)
    _, fp = _arr(F)
    for rec in r["flux"]:
        cn, cp = _cell(rec[:78]), _cell(rec[78:156])
        fc, fcp = _arr(rec[156:159])
        lib.ro_flux(ctypes.byref(m), ctypes.byref(cn), ctypes.byref(cp), fcp, rec[159], rec[160], rec[161],
                    int(rec[162]), fp)
        assert np.array_equal(F[:NFL], rec[163:163 + NFL], equal_nan=True), (F[:NFL], rec[163:163 + NFL])
    for rec in r["bflux"]:
        c = _cell(rec[:78])
        b = RoBc(int(rec[78]), tuple(rec[79:86]), tuple(rec[86:89]), rec[89])
        lib.ro_boundary_flux(ctypes.byref(m), ctypes.byref(b), ctypes.byref(c), rec[90], rec[91], rec[92],
                             int(rec[93]), int(rec[94]), fp)
        assert np.array_equal(F[:NFL], rec[95:95 + NFL], equal_nan=True), (int(rec[78]), F[:NFL], rec[95:95 + NFL])
    out = np.zeros(7)
    _, op = _arr(out)
    for rec in r["cell"]:
        c = _cell(rec[:78])
        u, up = _arr(rec[5:12])
        p, pp = _arr(rec[12:19])
        lib.ro_prim_from_cons(ctypes.byref(m), up, op)
        assert np.array_equal(out[:E], rec[89:89 + E])
        lib.ro_cons_from_prim(ctypes.byref(m), pp, op)
        assert np.array_equal(out[:E], rec[96:96 + E])
        assert lib.ro_max_delta_time(ctypes.byref(m), ctypes.byref(c)) == rec[103]
        c2 = _cell(rec[:78])
        lib.ro_compute_rhs(ctypes.byref(m), ctypes.byref(c2))
        assert np.array_equal(np.array(c2.data[19:19 + E]), rec[104:104 + E])
        du, dup = _arr(rec[78:89])
        lib.ro_source(ctypes.byref(m), ctypes.byref(c), dup, op)
        if m.model == 2:
            assert np.array_equal(out[:E], rec[111:111 + E])
        if G:
            g = np.zeros(6)
            _, gp = _arr(g)
            lib.ro_grad_input(ctypes.byref(m), pp, gp)
            assert np.array_equal(g[:G], rec[118:118 + G])
    for rec in r["lim"]:
        got = [lib.ro_limit(k, rec[0], rec[1]) for k in range(7)]
        assert np.array_equal(np.array(got), rec[2:9], equal_nan=True)
    for rec in r["est"]:
        c = _cell(rec[:78])
        w, wp = _arr(rec[78:85])
        nb, nbp = _arr(rec[85:127])
        pres = (ctypes.c_int * 6)(*[int(x) for x in rec[127:133]])
        assert lib.ro_estimate(ctypes.byref(m), wp, ctypes.byref(c), nbp, pres) == rec[133]
