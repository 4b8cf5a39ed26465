"""The simulation loop of DACTI's default_driver (driver/default_driver.hpp:77-217) over the GPU solver.

`run()` advances global steps until `end_time` (or a converged steady state), calling `integrate` with
`signal = time > signal_time`; after every step it decides, as the reference does, whether to write a
frame (simulation time advanced by at least `io_interval` since the last one, convergence, or NaN), and
then appends a row (time, frame, step, n_cells and the observers' integral variables) to
`<out_dir>/<name>_observables.csv` and writes `<out_dir>/<name>_<frame:04>.vtu` (vtu_writer, the
default) or `<out_dir>/<name>_<frame:04>.htg` (htg_writer, `writer="htg"`). Frame 0 is the initial
state. A NaN (force_break) ends the run after its frame, as in the reference.
"""
from __future__ import annotations

import os
import time as _time
from typing import Optional, Sequence

import numpy as np

from .htg import write_frame
from .io import write_vtu
from .solver import Solver


def _row(vals) -> str:
    """One CSV row; floats (numpy scalars included) in shortest round-trip form, integers as they are."""
    out = []
    for v in vals:
        if isinstance(v, (int, np.integer)) and not isinstance(v, bool):
            out.append(str(int(v)))
        else:
            out.append(repr(float(v)))
    return ",".join(out) + "\n"


class Totals:
    """Integral observer: conserved totals sum(u * volume) per component, named u_0 .. u_{E-1}."""

    name = "Totals"

    def __init__(self, E: int):
        self.names = [f"u_{q}" for q in range(E)]

    def observe(self, solver, snap) -> list:
        vol = (solver.side_length * 0.5 ** snap.tree_level.astype(np.float64)) ** snap.dims
        return list((snap.u * vol[:, None]).sum(axis=0))


class DropEnergy:
    """DACTI's DropEnergy observer (driver/observer/drop_energy.hpp:8-34) for the multiphase model:
    ke = sum vol 0.5 rho |v|^2 and Etot = sum vol (0.5 rho |v|^2 + sigma |grad alpha|), rho = p0 + p1,
    with |grad alpha| from the cell's stored volume-fraction gradient along x and y only (as the
    reference, also in 3D). The gradients come from dg_read_gradients, so the case needs viscous or
    conduction terms (the steps skip the gradient computation otherwise)."""

    name = "Droplet Energy"
    names = ["ke", "Etot"]

    def observe(self, solver, snap) -> list:
        sh = solver.shape
        D, iu, da = sh.dims, sh.iu, sh.dims + 1
        grad = solver.active_gradients()
        vol = (solver.side_length * 0.5 ** snap.tree_level.astype(np.float64)) ** D
        rho = snap.p[:, 0] + snap.p[:, 1]
        v2 = (snap.p[:, iu:iu + D] ** 2).sum(axis=1)
        norm = np.sqrt(grad[:, 0, da] ** 2 + grad[:, 1, da] ** 2)
        ke = vol * 0.5 * rho * v2
        return [float(ke.sum()), float((ke + vol * solver.params.sigma * norm).sum())]


def locate(snap, side_length: float, pts: np.ndarray) -> np.ndarray:
    """Integrator::get_cell_index (integrator/integrator.hpp:168) over the active leaves of `snap`:
    the row of the leaf containing each point, -1 where none does."""
    from .casefile import cell_coords

    lv = snap.tree_level.astype(np.int64)
    coords = cell_coords(snap.center, lv, side_length)
    D = snap.dims

    def key(level, c):
        k = np.asarray(level, np.int64) << np.int64(60)
        for d in range(D):
            k = k | (c[:, d].astype(np.int64) << np.int64(40 - 20 * d))
        return k

    keys = key(lv, coords)
    order = np.argsort(keys)
    sk = keys[order]
    out = np.full(pts.shape[0], -1, np.int64)
    for l in np.unique(lv):
        n_l = np.int64(1) << np.int64(l)
        pc = np.floor((pts[:, :D] / side_length + 0.5) * n_l).astype(np.int64)
        q = key(np.full(pts.shape[0], l), pc)
        pos = np.clip(np.searchsorted(sk, q), 0, sk.size - 1)
        hit = (sk[pos] == q) & (out < 0)
        out[hit] = order[pos[hit]]
    return out


def find_in_tree(nodes, side_length: float, active_size, periodic, pts: np.ndarray) -> np.ndarray:
    """Domain::find(p, max_depth) (integrator/domain.hpp:64-80, 407-416) over a whole node table: the
    slot of the leaf (active or not) containing each point, 0 for a point outside a non-periodic side of
    the active box. The descent picks child bit d when the point lies strictly above the centre."""
    D = nodes.dims
    root = nodes.root()
    act = np.asarray(active_size, np.float64)[:D]
    out = np.zeros(pts.shape[0], np.int64)
    for k in range(pts.shape[0]):
        x = np.array(pts[k, :D], np.float64)
        inside = True
        for d in range(D):
            if x[d] < -0.5 * act[d] or x[d] > 0.5 * act[d]:
                if periodic[d]:
                    x[d] = x[d] + act[d] if x[d] < -0.5 * act[d] else x[d] - act[d]
                else:
                    inside = False
        if not inside:
            continue
        x = 2.0 * x / side_length
        idx = root
        while idx != 0 and not (nodes.flags[idx] & 1):
            i = 0
            for d in range(D):
                if x[d] > 0.0:
                    i |= 1 << d
            q = np.array([1.0 if (i >> d) & 1 else -1.0 for d in range(D)])
            x = (x - 0.5 * q) * 2.0
            idx = int(nodes.children[idx, i])
        out[k] = idx
    return out


class AeroForce:
    """DACTI's AeroForce observer (driver/observer/aero_force.hpp:8-131) for 2D cases with analytic
    solid objects: pressure coefficients Cp = (p - p_ref) / (rho_ref |v_ref|^2 / 2) sampled along each
    object's outline, integrated to Cl and Cd; field variables Cp and ObjectSurface on the cells next to an
    object.

    convention="reference" (the default) follows aero_force.hpp:37-62 and 83-100: each outline segment
    a-b (the outline in the order its curve is sampled, counter-clockwise for circles and ellipses,
    scene/geometry_data.cpp:103-135) is split into max(int(10 |ab|), 1) samples at a + (j + 0.5) ab / n,
    each moved by -0.01 n_s with n_s = rotaten90(ab / |ab|) = (ab_y, -ab_x) / |ab| (into the body for a
    counter-clockwise outline); the sample's cell is Domain::find over the whole tree, inactive leaves
    included (Integrator::get_cell_index, integrator.hpp:168), so samples inside a body read that
    leaf's stored state; Cl = sum Cp area n_s,y and Cd = sum Cp area n_s,x. The outline is the analytic
    curve cut into `n_segments` pieces instead of the adaptively sampled mesh.

    convention="fluid" moves the samples 0.01 into the fluid, locates them among the active cells, and
    reports the pressure force on the body per unit span and dynamic pressure with drag positive along
    +x: a physical reading of the same quantities, not the reference's numbers."""

    name = "Aerodynamic Forces"
    names = ["Cl", "Cd"]
    field_names = ["Cp", "ObjectSurface"]

    def __init__(self, objects, p_ref, vel_ref, n_segments: int = 256, sample_resolution: int = 10,
                 convention: str = "reference"):
        if convention not in ("reference", "fluid"):
            raise ValueError("convention is 'reference' or 'fluid'")
        self.convention = convention
        self.objects = list(objects)  # every object is sampled, as in the reference
        self.walls = [o for o in self.objects if getattr(o, "bc", None) is not None]
        self.p_ref = np.asarray(p_ref, np.float64)
        v = np.asarray(vel_ref, np.float64)
        self.q_inv = 2.0 / (self.p_ref[0] * float(v @ v))
        pts, area, nrm = [], [], []
        for o in self.objects:
            ring = o.outline(n_segments)
            nxt = np.roll(ring, -1, axis=0)
            for a, b in zip(ring, nxt):
                ab = b - a
                length = float(np.hypot(*ab))
                n_s = np.array([ab[1], -ab[0]]) / length  # rotaten90 of the unit tangent
                k = max(int(sample_resolution * length), 1)
                for j in range(k):
                    pos = a + (j + 0.5) * ab / k
                    pts.append(pos - 0.01 * n_s if convention == "reference" else pos + 0.01 * n_s)
                    area.append(length / k)
                    nrm.append(n_s)
        self.pts, self.area, self.nrm = np.array(pts), np.array(area), np.array(nrm)

    def observe(self, solver, snap) -> list:
        ip = solver.shape.ip
        if self.convention == "reference":
            nodes = solver.tree_nodes()
            prm = solver.params
            idx = find_in_tree(nodes, solver.side_length, prm.active_size, prm.periodic, self.pts)
            cp = (nodes.p[idx, ip] - self.p_ref[ip]) * self.q_inv
            cl = float((cp * self.area * self.nrm[:, 1]).sum())
            cd = float((cp * self.area * self.nrm[:, 0]).sum())
            return [cl, cd]
        idx = locate(snap, solver.side_length, self.pts)
        ok = idx >= 0
        cp = np.zeros(idx.size)
        cp[ok] = (snap.p[idx[ok], ip] - self.p_ref[ip]) * self.q_inv
        fx = -(cp * self.area * self.nrm[:, 0]).sum()
        fy = -(cp * self.area * self.nrm[:, 1]).sum()
        return [float(fy), float(fx)]

    def fields(self, solver, snap) -> list:
        D = snap.dims
        size = solver.side_length * 0.5 ** snap.tree_level.astype(np.float64)
        surf = np.zeros(snap.n, bool)
        for d in range(D):
            for sgn in (-1.0, 1.0):
                c = snap.center.copy()
                c[:, d] += sgn * size
                for o in self.walls:
                    surf |= o.signed_distance(c) < 0.0
        ip = solver.shape.ip
        cp = np.where(surf, (snap.p[:, ip] - self.p_ref[ip]) * self.q_inv, 0.0)
        return [cp, surf.astype(np.float64)]


class DefaultDriver:
    def __init__(self, solver: Solver, name: str, out_dir: str, end_time: Optional[float] = None,
                 io_interval: float = 0.0, observers: Sequence = (), convergence_tol: float = 0.0,
                 signal_time: float = 0.0, write_frames: bool = True, max_steps: Optional[int] = None,
                 writer: str = "vtu"):
        if writer not in ("vtu", "htg"):
            raise ValueError("writer is 'vtu' (vtu_writer) or 'htg' (htg_writer)")
        self.writer = writer
        self.s, self.name, self.out_dir = solver, name, out_dir
        self.end_time, self.io_interval = end_time, io_interval
        self.observers, self.convergence_tol, self.signal_time = list(observers), convergence_tol, signal_time
        self.write_frames, self.max_steps = write_frames, max_steps
        self.log: list = []

    def _observe(self, snap) -> list:
        vals = []
        for ob in self.observers:
            vals += ob.observe(self.s, snap)
        return vals

    def _frame(self, frame: int, snap) -> None:
        if self.write_frames and self.writer == "htg":
            # htg_writer takes the observers' fields and does not write them (htg_writer.hpp:27-33)
            write_frame(self.out_dir, self.name, frame, self.s.tree_nodes(), float(self.s.params.active_size[0]))
        elif self.write_frames:
            # observers' field variables as cell data "<observer>/<field>" (driver/default_driver.hpp:45-72)
            fields = {}
            for ob in self.observers:
                if hasattr(ob, "fields"):
                    for fname, arr in zip(ob.field_names, ob.fields(self.s, snap)):
                        fields[f"{ob.name}/{fname}"] = arr
            write_vtu(os.path.join(self.out_dir, f"{self.name}_{frame:04d}.vtu"), snap, self.s.active_slopes(),
                      self.s.side_length, fields=fields)

    def run(self) -> dict:
        os.makedirs(self.out_dir, exist_ok=True)
        t_start = _time.perf_counter()
        names = [n for ob in self.observers for n in ob.names]
        csv = open(os.path.join(self.out_dir, f"{self.name}_observables.csv"), "w")
        csv.write("time,frame,step," + ",".join(["n_cells"] + names) + "\n")
        snap = self.s.active_cells()
        integ = self._observe(snap)
        self._frame(0, snap)
        sim_time, last_print, frame, step, last_step = 0.0, 0.0, 0, 0, 0
        converged = force_break = False
        while (self.end_time is None or sim_time < self.end_time) and not converged:
            if self.max_steps is not None and step >= self.max_steps:
                break
            gdt, force_break = self.s.integrate(signal=sim_time > self.signal_time)
            sim_time += gdt
            snap = None
            if self.convergence_tol > 0:
                snap = self.s.active_cells()
                old, integ = integ, self._observe(snap)
                csv.write(_row([sim_time, frame, step, snap.n] + integ))
                delta = max((abs(a - b) / gdt for a, b in zip(integ, old)), default=0.0)
                converged = delta < self.convergence_tol
            if sim_time - last_print >= self.io_interval or converged or force_break:
                frame += 1
                snap = snap or self.s.active_cells()
                integ = self._observe(snap)
                csv.write(_row([sim_time, frame, step, snap.n] + integ))
                csv.flush()
                self.log.append({"frame": frame, "time": sim_time, "steps": step - last_step, "cells": snap.n,
                                 "global_dt": gdt, "seconds": _time.perf_counter() - t_start})
                last_print, last_step = sim_time, step
                self._frame(frame, snap)
            if force_break:
                break
            step += 1
        csv.close()
        return {"time": sim_time, "steps": step, "frames": frame, "force_break": bool(force_break),
                "converged": converged}
