"""Python binding of the C ABI (include/dacti_gpu.h), shaped like DACTI's Integrator.

``Solver(case)`` runs the Integrator constructor (integrator/integrator.hpp:72-163) on the device,
``integrate()`` advances one global step like Integrator::integrate (impl/integrate.hpp:12-87),
``n_active_cells()`` and ``active_cells()`` mirror n_active_cells / for_each_active_cell
(integrator/integrator.hpp:172-202). There is no CPU fallback: without the compiled library or a
CUDA device, construction raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Callable, Optional

import numpy as np

from .casefile import Case, Snapshot
from .htg import NodeTable

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdacti_gpu.so")

DG_OK = 0
STATUS_NAMES = {
    -1: "DG_ERR_ARG", -2: "DG_ERR_CUDA", -3: "DG_ERR_CAPACITY", -4: "DG_ERR_DEPTH", -5: "DG_ERR_MISSING_BC",
    -6: "DG_ERR_UNSUPPORTED",
}

LIMITERS = {"minmod": 0, "unlimited": 1, "van_leer": 2, "superbee": 3, "von_alba_2": 4, "koren": 5,
            "first_order": 6}


class DgCase(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("dims", ctypes.c_int), ("n_nodes", ctypes.c_int), ("n_bc", ctypes.c_int),
        ("n_zones", ctypes.c_int), ("limiter", ctypes.c_int),
        ("params", ctypes.POINTER(ctypes.c_double)), ("weights", ctypes.POINTER(ctypes.c_double)),
        ("zones", ctypes.POINTER(ctypes.c_double)), ("bc_type", ctypes.POINTER(ctypes.c_int)),
        ("bc_p_in", ctypes.POINTER(ctypes.c_double)), ("bc_normal", ctypes.POINTER(ctypes.c_double)),
        ("bc_fade_in", ctypes.POINTER(ctypes.c_double)), ("parent", ctypes.POINTER(ctypes.c_int)),
        ("children", ctypes.POINTER(ctypes.c_int)), ("level", ctypes.POINTER(ctypes.c_int)),
        ("flags", ctypes.POINTER(ctypes.c_uint)), ("bc", ctypes.POINTER(ctypes.c_int)),
        ("center", ctypes.POINTER(ctypes.c_double)), ("p", ctypes.POINTER(ctypes.c_double)),
    ]


class DgStats(ctypes.Structure):
    _fields_ = [
        ("n_clusters", ctypes.c_longlong * 16), ("n_buffers", ctypes.c_longlong * 16),
        ("tree_size", ctypes.c_longlong), ("n_splits", ctypes.c_longlong), ("n_unsplits", ctypes.c_longlong),
        ("n_gc", ctypes.c_longlong), ("n_substeps", ctypes.c_longlong), ("n_global_steps", ctypes.c_longlong),
        ("cell_updates", ctypes.c_longlong), ("max_acti_level", ctypes.c_int), ("global_dt", ctypes.c_double),
        ("acti_time", ctypes.c_double * 16), ("acti_counter", ctypes.c_int * 16),
        ("n_launches", ctypes.c_longlong), ("kernel_ms", ctypes.c_double * 12),
        ("kernel_launches", ctypes.c_longlong * 12), ("kernel_cells", ctypes.c_longlong * 12),
    ]


KERNEL_KINDS = ("flux", "recv", "update", "slope", "aux", "estimate", "regrid", "reassign", "flush", "init", "gc",
                "other")


SUBSTEP_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                              ctypes.c_longlong)

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the compiled library; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m dacti_b200.build`")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.dg_create.argtypes = [ctypes.POINTER(DgCase), ctypes.POINTER(vp)]
    lib.dg_set_device.argtypes = [ctypes.c_int]
    lib.dg_set_stream.argtypes = [vp, vp]
    lib.dg_step.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                            SUBSTEP_FN, vp]
    lib.dg_step_many.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    lib.dg_cell_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.dg_read_cells.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                  ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    lib.dg_read_cells_noalloc.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                          ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]
    lib.dg_read_slopes.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.c_longlong,
                                   ctypes.POINTER(ctypes.c_longlong)]
    lib.dg_read_gradients.argtypes = lib.dg_read_slopes.argtypes
    lib.dg_forecast_features.argtypes = lib.dg_read_slopes.argtypes
    fp, dp, ll = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.c_longlong
    lib.dg_set_hold.argtypes = [vp, ctypes.POINTER(ctypes.c_ubyte), ll]
    lib.dg_set_coarsen_interval.argtypes = [vp, ctypes.c_int]
    ip, up = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint)
    lib.dg_tree_size.argtypes = [vp, ctypes.POINTER(ll)]
    lib.dg_read_tree.argtypes = [vp, ip, ip, ip, up, dp, dp, ll, ctypes.POINTER(ll)]
    lib.dg_mlp_last_error.argtypes = []
    lib.dg_mlp_last_error.restype = ctypes.c_char_p
    lib.dg_mlp_create.argtypes = [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(vp)]
    lib.dg_mlp_param_count.argtypes = [vp, ctypes.POINTER(ll)]
    lib.dg_mlp_set_params.argtypes = [vp, fp]
    lib.dg_mlp_get_params.argtypes = [vp, fp]
    lib.dg_mlp_predict.argtypes = [vp, fp, ll, fp]
    lib.dg_mlp_loss_grad.argtypes = [vp, fp, fp, ll, ctypes.c_float, fp, dp]
    lib.dg_mlp_train.argtypes = [vp, fp, fp, ll, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                 ctypes.c_ulonglong, dp]
    lib.dg_mlp_destroy.argtypes = [vp]
    lib.dg_get_stats.argtypes = [vp, ctypes.POINTER(DgStats)]
    lib.dg_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.dg_set_form.argtypes = [vp, ctypes.c_int]
    lib.dg_set_options.argtypes = [vp, ctypes.c_int]
    lib.dg_last_error.argtypes = [vp]
    lib.dg_last_error.restype = ctypes.c_char_p
    lib.dg_destroy.argtypes = [vp]
    lib.dg_destroy.restype = None
    lib.dg_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
    lib.dg_batch_step.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    lib.dg_batch_last_error.argtypes = [vp]
    lib.dg_batch_last_error.restype = ctypes.c_char_p
    lib.dg_batch_destroy.argtypes = [vp]
    lib.dg_batch_destroy.restype = None
    lib.dg_batch_set_launch.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    lib.dg_batch_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.dg_batch_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.c_int]
    lib.dg_batch_run_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    lib.dg_batch_set_pregrow.argtypes = [vp, ctypes.c_int]
    _lib = lib
    return lib


EXPORTED_SYMBOLS = ("dg_set_device", "dg_create", "dg_set_stream", "dg_step", "dg_step_many", "dg_cell_count",
                    "dg_read_cells", "dg_read_slopes", "dg_read_gradients", "dg_forecast_features", "dg_set_hold", "dg_set_coarsen_interval",
                    "dg_tree_size", "dg_read_tree",
                    "dg_mlp_last_error", "dg_mlp_create", "dg_mlp_param_count", "dg_mlp_set_params",
                    "dg_mlp_get_params", "dg_mlp_predict", "dg_mlp_loss_grad", "dg_mlp_train", "dg_mlp_destroy",
                    "dg_build_last_error", "dg_build_tree", "dg_tree_nodes", "dg_tree_copy", "dg_tree_free",
                    "dg_read_cells_noalloc", "dg_get_stats", "dg_batch_create", "dg_batch_step",
                    "dg_batch_last_error", "dg_batch_destroy", "dg_batch_set_launch", "dg_batch_set_profiling",
                    "dg_batch_stage_times", "dg_batch_run_stats", "dg_batch_set_pregrow",
                    "dg_set_form", "dg_set_options", "dg_set_profiling", "dg_last_error", "dg_destroy")

# Stage implementation choices (DG_OPT_* in dacti_gpu.h); every combination gives the same bits.
OPT_ORDERED_LISTS = 1
OPT_FACE_TILES = 2
OPT_DEFAULT = OPT_ORDERED_LISTS | OPT_FACE_TILES


class DgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Solver:
    def __init__(self, case: Case, limiter: Optional[str] = None, device: int = 0):
        self._lib = load_library()
        self._check_plain(self._lib.dg_set_device(device))
        t, prm = case.tree, case.params
        sh = t.shape
        self.shape = sh
        self.side_length = prm.side_length
        self.params = prm
        E, D = sh.E, sh.dims
        nb = max(len(t.bcs), 1)
        keep = dict(
            params=prm.param_vector(),
            weights=np.ascontiguousarray(prm.weights, np.float64).reshape(E),
            zones=np.array([[*(list(z.x0) + [0.0] * 3)[:3], *(list(z.x1) + [0.0] * 3)[:3], float(z.level)]
                            for z in prm.zones] or [[0.0] * 7], np.float64),
            bc_type=np.array([int(b.type) for b in t.bcs] or [0], np.int32),
            bc_p_in=np.array([list(b.p_in) for b in t.bcs] or [[0.0] * E], np.float64).reshape(nb, E),
            bc_normal=np.array([list(b.normal) for b in t.bcs] or [[0.0] * D], np.float64).reshape(nb, D),
            bc_fade_in=np.array([b.fade_in for b in t.bcs] or [0.0], np.float64),
            parent=np.ascontiguousarray(t.parent, np.int32),
            children=np.ascontiguousarray(t.children, np.int32),
            level=np.ascontiguousarray(t.level, np.int32),
            flags=np.ascontiguousarray(t.flags, np.uint32),
            bc=np.ascontiguousarray(t.bc, np.int32),
            center=np.ascontiguousarray(t.center, np.float64),
            p=np.ascontiguousarray(t.p, np.float64),
        )
        c = DgCase()
        c.model, c.dims, c.n_nodes = int(sh.model), D, t.n_nodes
        lim_id = LIMITERS[limiter] if limiter is not None else int(prm.limiter)
        c.n_bc, c.n_zones, c.limiter = len(t.bcs), len(prm.zones), lim_id
        dbl, it = ctypes.c_double, ctypes.c_int
        c.params, c.weights, c.zones = _ptr(keep["params"], dbl), _ptr(keep["weights"], dbl), _ptr(keep["zones"], dbl)
        c.bc_type, c.bc_p_in = _ptr(keep["bc_type"], it), _ptr(keep["bc_p_in"], dbl)
        c.bc_normal, c.bc_fade_in = _ptr(keep["bc_normal"], dbl), _ptr(keep["bc_fade_in"], dbl)
        c.parent, c.children, c.level = _ptr(keep["parent"], it), _ptr(keep["children"], it), _ptr(keep["level"], it)
        c.flags, c.bc = _ptr(keep["flags"], ctypes.c_uint), _ptr(keep["bc"], it)
        c.center, c.p = _ptr(keep["center"], dbl), _ptr(keep["p"], dbl)
        h = ctypes.c_void_p()
        rc = self._lib.dg_create(ctypes.byref(c), ctypes.byref(h))
        if rc != DG_OK:
            raise DgError(rc, self._lib.dg_last_error(None).decode())
        self._h = h
        self.global_dt = self.stats().global_dt
        self.time = 0.0

    # -- reference Integrator surface ---------------------------------------------------------
    def integrate(self, substep_hook: Optional[Callable] = None, signal: bool = True) -> tuple:
        """One global step. Returns (global_dt, force_break)."""
        fb = ctypes.c_int(0)
        gdt = ctypes.c_double(0.0)
        if substep_hook is not None:
            def tramp(_u, level, at, ns, dtl, csize):
                substep_hook(self, level, at, ns, dtl, csize)
            cb = SUBSTEP_FN(tramp)
        else:
            cb = SUBSTEP_FN()
        self._check(self._lib.dg_step(self._h, 1 if signal else 0, ctypes.byref(fb), ctypes.byref(gdt), cb, None))
        self.global_dt = gdt.value
        return gdt.value, bool(fb.value)

    def n_active_cells(self) -> int:
        n = ctypes.c_longlong()
        self._check(self._lib.dg_cell_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def active_cells(self) -> Snapshot:
        return self._read(self._lib.dg_read_cells)

    def _read(self, fn) -> Snapshot:
        sh = self.shape
        D, E = sh.dims, sh.E
        W = D + 1 + 2 * E + 3 + sh.P
        n = self.n_active_cells()
        lv = np.zeros((max(n, 1), 2), np.int32)
        data = np.zeros((max(n, 1), W), np.float64)
        got = ctypes.c_longlong()
        self._check(fn(self._h, _ptr(lv, ctypes.c_int), _ptr(data, ctypes.c_double), n, ctypes.byref(got)))
        st = self.stats()
        n_in = int(sum(st.n_clusters))
        return Snapshot(
            D, E, int(st.n_global_steps), int(st.n_substeps), int(st.tree_size), n_in, self.time, st.global_dt,
            float(st.cell_updates), lv[:n, 0].copy(), lv[:n, 1].copy(), data[:n, :D].copy(), data[:n, D].copy(),
            data[:n, D + 1:D + 1 + E].copy(), data[:n, D + 1 + E:D + 1 + 2 * E].copy(), data[:n, D + 1 + 2 * E].copy(),
            data[:n, D + 2 + 2 * E].copy(), data[:n, D + 3 + 2 * E].copy(),
            data[:n, D + 4 + 2 * E:].copy() if sh.P > 0 else None,
        )

    def active_cells_noalloc(self) -> Snapshot:
        """active_cells() through dg_read_cells_noalloc: no device allocation (bounded scratch)."""
        return self._read(self._lib.dg_read_cells_noalloc)

    def active_slopes(self) -> np.ndarray:
        """dg_read_slopes: the active cells' limited slopes, shape (n, D, E), in active_cells() order."""
        sh = self.shape
        n = self.n_active_cells()
        out = np.zeros((max(n, 1), sh.dims, sh.E))
        got = ctypes.c_longlong(0)
        self._check(self._lib.dg_read_slopes(self._h, _ptr(out, ctypes.c_double), n, ctypes.byref(got)))
        return out[: got.value]

    def active_gradients(self) -> np.ndarray:
        """dg_read_gradients: the active cells' gradients of the gradient inputs, shape (n, D, G), in
        active_cells() order (Navier-Stokes and viscous multiphase cases only)."""
        sh = self.shape
        n = self.n_active_cells()
        out = np.zeros((max(n, 1), sh.dims, sh.G))
        got = ctypes.c_longlong(0)
        self._check(self._lib.dg_read_gradients(self._h, _ptr(out, ctypes.c_double), n, ctypes.byref(got)))
        return out[: got.value]

    def forecast_features(self) -> np.ndarray:
        """dg_forecast_features: the regrid forecaster's inputs, shape (n, 5 + 5D), float32, in
        active_cells() order."""
        sh = self.shape
        n = self.n_active_cells()
        F = 5 + 5 * sh.dims
        out = np.zeros((max(n, 1), F))
        got = ctypes.c_longlong(0)
        self._check(self._lib.dg_forecast_features(self._h, _ptr(out, ctypes.c_double), n, ctypes.byref(got)))
        return out[: got.value].astype(np.float32)

    def tree_nodes(self) -> NodeTable:
        """dg_read_tree: every node slot of the device pool (Integrator::get_nodes), what the HTG writer
        walks. Slot numbers are the device's; the tree they link is the reference's."""
        sh = self.shape
        n = ctypes.c_longlong(0)
        self._check(self._lib.dg_tree_size(self._h, ctypes.byref(n)))
        n = int(n.value)
        C = 1 << sh.dims
        parent = np.zeros(max(n, 1), np.int32)
        children = np.zeros((C, max(n, 1)), np.int32)
        level = np.zeros(max(n, 1), np.int32)
        flags = np.zeros(max(n, 1), np.uint32)
        p = np.zeros((sh.E, max(n, 1)))
        meta = np.zeros((4, max(n, 1)))
        got = ctypes.c_longlong(0)
        self._check(self._lib.dg_read_tree(self._h, _ptr(parent, ctypes.c_int), _ptr(children, ctypes.c_int),
                                           _ptr(level, ctypes.c_int), _ptr(flags, ctypes.c_uint),
                                           _ptr(p, ctypes.c_double), _ptr(meta, ctypes.c_double), n,
                                           ctypes.byref(got)))
        # the device copies component-major rows of exactly n values each
        k = int(got.value)
        children = children.reshape(-1)[: C * k].reshape(C, k)
        p = p.reshape(-1)[: sh.E * k].reshape(sh.E, k)
        meta = meta.reshape(-1)[: 4 * k].reshape(4, k)
        return NodeTable(sh.dims, parent[:k].copy(), np.ascontiguousarray(children.T), level[:k].copy(),
                         flags[:k].copy(), np.ascontiguousarray(p.T), np.ascontiguousarray(meta.T))

    def set_hold(self, hold) -> None:
        """dg_set_hold: one flag per active cell (active_cells() order)."""
        h = np.ascontiguousarray(hold, np.uint8)
        self._check(self._lib.dg_set_hold(self._h, h.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), h.size))

    def set_coarsen_interval(self, steps: int) -> None:
        self._check(self._lib.dg_set_coarsen_interval(self._h, steps))

    def stats(self) -> DgStats:
        s = DgStats()
        self._check(self._lib.dg_get_stats(self._h, ctypes.byref(s)))
        return s

    def set_form(self, form: str) -> None:
        """'fp64' (the reference's arithmetic) or 'mixed' (FP32 reconstruction and flux, FP64 update)."""
        self._check(self._lib.dg_set_form(self._h, {"fp64": 0, "mixed": 1}[form]))

    def set_options(self, options: int) -> None:
        """Stage implementation choices: OPT_ORDERED_LISTS, OPT_FACE_TILES (OPT_DEFAULT at creation)."""
        self._check(self._lib.dg_set_options(self._h, int(options)))

    def set_profiling(self, on: bool = True) -> None:
        self._check(self._lib.dg_set_profiling(self._h, 1 if on else 0))

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self._lib.dg_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_plain(self, rc: int) -> None:
        if rc != DG_OK:
            raise DgError(rc, "invalid device")

    def _check(self, rc: int) -> None:
        if rc != DG_OK:
            raise DgError(rc, self._lib.dg_last_error(self._h).decode())


def step_many(solvers, threads: int = 32, signal: bool = True) -> list:
    """dg_step_many: one global step of every solver, concurrently (host threads, one stream each).
    Returns the force_break flags; raises DgError with the first failing solver's message."""
    lib = load_library()
    n = len(solvers)
    if n == 0:
        return []
    hs = (ctypes.c_void_p * max(n, 1))(*[s._h for s in solvers])
    fb = (ctypes.c_int * max(n, 1))()
    gdt = (ctypes.c_double * max(n, 1))()
    st = (ctypes.c_int * max(n, 1))()
    rc = lib.dg_step_many(hs, n, threads, 1 if signal else 0, fb, gdt, st)
    if rc != 0:
        for k in range(n):
            if st[k] != 0:
                raise DgError(st[k], lib.dg_last_error(solvers[k]._h).decode())
        raise DgError(rc, "dg_step_many failed")
    return [bool(fb[k]) for k in range(n)]


BATCH_STAGES = ("face_sum", "receive", "update", "slope", "aux", "estimate", "regrid_cell", "regrid_fresh",
                "nbr_list", "flush")


def step_batches(batches) -> list:
    """One global step of several lockstep batches at once, one host thread each (every batch has its own
    stream, and ctypes releases the GIL during the call), so the batches' kernels overlap on the GPU.
    Returns the force_break flags of every batch's trees, batch by batch."""
    from concurrent.futures import ThreadPoolExecutor
    if len(batches) == 1:
        return [batches[0].step()]
    with ThreadPoolExecutor(max_workers=len(batches)) as ex:
        return list(ex.map(lambda b: b.step(), batches))


class Batch:
    """dg_batch: independent solvers of one model stepped in lockstep, one launch per stage for all trees
    that run a level (merged ACTI schedules). Per tree the results equal Solver.integrate's bit for bit.
    The solvers stay usable for read-backs; step them through the batch only, and close the batch before
    closing them. `launch` (blocks per SM per stage kind) defaults to the autotuned table of the model
    when dacti_b200/launch_table.json has one."""

    def __init__(self, solvers, launch=None):
        self._lib = load_library()
        self.solvers = list(solvers)
        hs = (ctypes.c_void_p * len(self.solvers))(*[s._h for s in self.solvers])
        h = ctypes.c_void_p()
        rc = self._lib.dg_batch_create(hs, len(self.solvers), ctypes.byref(h))
        if rc != DG_OK:
            raise DgError(rc, self._lib.dg_batch_last_error(None).decode())
        self._h = h
        if launch is None:
            from .autotune import table_entry
            launch = table_entry(self.solvers[0].shape)
        if launch is not None:
            self.set_launch(launch)

    def _bcheck(self, rc: int) -> None:
        if rc != DG_OK:
            raise DgError(rc, self._lib.dg_batch_last_error(self._h).decode())

    def set_launch(self, blocks_per_sm) -> None:
        v = (ctypes.c_int * len(blocks_per_sm))(*[int(x) for x in blocks_per_sm])
        self._bcheck(self._lib.dg_batch_set_launch(self._h, v, len(blocks_per_sm)))

    def set_profiling(self, on: bool = True) -> None:
        self._bcheck(self._lib.dg_batch_set_profiling(self._h, 1 if on else 0))

    def stage_times(self) -> dict:
        """{stage: (device ms, work items)} since the previous call (profiling on)."""
        n = len(BATCH_STAGES)
        ms = (ctypes.c_double * n)()
        it = (ctypes.c_longlong * n)()
        self._bcheck(self._lib.dg_batch_stage_times(self._h, ms, it, n))
        return {k: (ms[i], it[i]) for i, k in enumerate(BATCH_STAGES)}

    def set_pregrow(self, on: bool = True) -> None:
        """Grow pools ahead of each planned run (default) or only where a run stops at the capacity check."""
        self._bcheck(self._lib.dg_batch_set_pregrow(self._h, 1 if on else 0))

    def run_stats(self) -> dict:
        """Planned runs (one per global step once warmed up, unless a check stopped one), runs a check
        stopped, substeps planned, and substeps the host completed after a stop at the capacity check,
        since the batch was made."""
        v = (ctypes.c_longlong * 4)()
        self._bcheck(self._lib.dg_batch_run_stats(self._h, v, 4))
        return {"runs": v[0], "stops": v[1], "planned": v[2], "completed": v[3]}

    def step(self, signal: bool = True) -> list:
        """One global step of every tree; returns the force_break flags."""
        n = len(self.solvers)
        fb = (ctypes.c_int * n)()
        gdt = (ctypes.c_double * n)()
        rc = self._lib.dg_batch_step(self._h, 1 if signal else 0, fb, gdt)
        if rc != DG_OK:
            raise DgError(rc, self._lib.dg_batch_last_error(self._h).decode())
        for k, s in enumerate(self.solvers):
            s.global_dt = gdt[k]
        return [bool(fb[k]) for k in range(n)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
