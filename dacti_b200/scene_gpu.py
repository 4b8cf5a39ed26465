"""Initial tree built on the GPU (dg_build_tree in csrc/scene_build.cu) from a SceneSpec.

Same nodes, in the same order, as scene.build_tree for the scenes it covers: spheres, ellipses and
polygons (droplets, bubbles and solids with their object boundaries and fix_boundary), domain-face boundaries,
refinement zones, the initial jump and inflow_r faces, a uniform or jump initial condition given as
data (`SceneSpec.ic`) and the tanh interface. The device marks object faces; their conditions and
normals are assigned here with the host builder's own rule, so only the numbering of the boundary
table can differ from scene.build_tree's. Polygons with more than 8 vertices or a programmatic-only
initial condition raise NotImplementedError; build those with scene.build_tree.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from .models import BcType
from .scene import BoundarySpec, EllipseObject, PolygonObject, SceneSpec, SphereObject, Tree, _ObjectBoundaries
from .solver import DG_OK, DgError, load_library

_D = ctypes.c_double
_I = ctypes.c_int


class DgScene(ctypes.Structure):
    _fields_ = [
        ("model", _I), ("dims", _I),
        ("side_length", _D), ("active_size", _D * 3),
        ("min_level", _I), ("max_level", _I), ("max_level_geom", _I),
        ("refinement_radius", _D),
        ("domain_bc", (_I * 2) * 3), ("inflow_r", (_I * 2) * 3),
        ("n_objects", _I), ("objects", ctypes.POINTER(_D)),
        ("n_zones", _I), ("zones", ctypes.POINTER(_D)),
        ("refine_jump", _I), ("jump_axis", _I), ("jump_location", _D),
        ("ic_kind", _I), ("ic_axis", _I), ("ic_location", _D),
        ("ic_neg", ctypes.POINTER(_D)), ("ic_pos", ctypes.POINTER(_D)),
        ("diffuse_ic", _I), ("keep_ic_gas_density", _I),
        ("rho_ref", _D * 2),
    ]


def _bind(lib):
    if getattr(lib, "_dg_build_bound", False):
        return lib
    vp = ctypes.c_void_p
    ip, up, dp = ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(_D)
    lib.dg_build_last_error.argtypes = []
    lib.dg_build_last_error.restype = ctypes.c_char_p
    lib.dg_build_tree.argtypes = [ctypes.POINTER(DgScene), ctypes.POINTER(vp)]
    lib.dg_tree_nodes.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    lib.dg_tree_copy.argtypes = [vp, ip, ip, ip, up, ip, dp, dp]
    lib.dg_tree_free.argtypes = [vp]
    lib._dg_build_bound = True
    return lib


MAX_VERT = 8


def _object_row(o) -> list:
    """One row of dg_scene.objects (29 values)."""
    kind = {"droplet": 0.0, "bubble": 1.0}.get(o.type, 2.0)
    has_bc = o.bc is not None
    inflow_r = has_bc and o.bc.type == BcType.INFLOW_R
    tail = [kind, 1.0 if has_bc else 0.0, 1.0 if inflow_r else 0.0]
    if isinstance(o, PolygonObject):
        v = np.asarray(o.vertices, np.float64)
        if v.shape[0] > MAX_VERT or v.shape[0] < 3 or v.shape[1] != 2:
            raise NotImplementedError("polygons with fewer than 3 or more than 8 vertices (lines included) need "
                                      "the host builder")
        verts = np.zeros((MAX_VERT, 2))
        verts[: v.shape[0]] = v
        return [0.0] * 6 + [1.0, 0.0, 2.0] + tail + [float(v.shape[0])] + list(verts.ravel())
    if not isinstance(o, (SphereObject, EllipseObject)):
        raise NotImplementedError(f"{type(o).__name__} objects need the host builder")
    c = list(np.asarray(o.center, np.float64)) + [0.0] * 3
    if isinstance(o, SphereObject):
        axes, cs, sn, shape = [o.radius, o.radius, o.radius], 1.0, 0.0, 0
    elif isinstance(o, EllipseObject):
        a = list(np.asarray(o.axes, np.float64)) + [1.0] * 3
        axes, shape = a[:3], 1
        if o.angle_deg != 0.0:
            th = o.angle_deg * math.pi / 180.0
            cs, sn = math.cos(th), math.sin(th)
        else:
            cs, sn = 1.0, 0.0
    else:
        raise NotImplementedError(f"{type(o).__name__} objects need the host builder")
    return c[:3] + axes + [cs, sn, float(shape)] + tail + [0.0] * (1 + 2 * MAX_VERT)


def build_tree_device(spec: SceneSpec) -> Tree:
    sh = spec.shape
    D, E = sh.dims, sh.E
    if spec.ic is None:
        raise NotImplementedError("the device builder needs the initial condition as data (SceneSpec.ic)")
    lib = _bind(load_library())
    sc = DgScene()
    sc.model, sc.dims = int(sh.model), D
    sc.side_length = spec.side_length
    for d in range(3):
        sc.active_size[d] = float(spec.active_size[d]) if d < D else 0.0
    sc.min_level, sc.max_level = spec.min_level, spec.max_level
    sc.max_level_geom = spec.max_level if spec.max_level_geom is None else spec.max_level_geom
    sc.refinement_radius = spec.refinement_radius
    # boundary table: domain faces first, in (dim, dir) order, as scene.build_tree numbers them
    bcs, k = [], 0
    for d in range(3):
        for side in range(2):
            sc.domain_bc[d][side] = -1
            sc.inflow_r[d][side] = 0
    for d in range(D):
        pair = spec.domain_bc[d]
        if pair is None:
            continue
        for side in range(2):
            b = pair[side]
            normal = [0.0] * D
            if b.type in (BcType.FREESLIP, BcType.NOSLIP):
                normal[d] = -(2.0 * side - 1.0)
            sc.domain_bc[d][side] = k
            sc.inflow_r[d][side] = 1 if b.type == BcType.INFLOW_R else 0
            bcs.append(BoundarySpec(b.type, list(b.p_in) if b.p_in is not None else [0.0] * E, normal, b.fade_in))
            k += 1
    objs = np.array([_object_row(o) for o in spec.objects] or [[0.0] * (13 + 2 * MAX_VERT)], np.float64)
    sc.n_objects = len(spec.objects)
    sc.objects = objs.ctypes.data_as(ctypes.POINTER(_D))
    zones = np.array([list(z.x0) + list(z.x1) + [float(z.level)] for z in spec.zones] or [[0.0] * 7], np.float64)
    sc.n_zones = len(spec.zones)
    sc.zones = zones.ctypes.data_as(ctypes.POINTER(_D))
    if spec.jump is not None:
        sc.refine_jump, sc.jump_axis, sc.jump_location = 1, int(spec.jump[0]), float(spec.jump[1])
    if spec.ic[0] == "uniform":
        neg = np.asarray(spec.ic[1], np.float64).reshape(E)
        pos = neg.copy()
        sc.ic_kind = 0
    elif spec.ic[0] == "jump":
        _, axis, loc, n_, p_ = spec.ic
        neg, pos = np.asarray(n_, np.float64).reshape(E), np.asarray(p_, np.float64).reshape(E)
        sc.ic_kind, sc.ic_axis, sc.ic_location = 1, int(axis), float(loc)
    else:
        raise ValueError(f"unknown initial condition kind {spec.ic[0]!r}")
    sc.ic_neg = neg.ctypes.data_as(ctypes.POINTER(_D))
    sc.ic_pos = pos.ctypes.data_as(ctypes.POINTER(_D))
    sc.diffuse_ic = 1 if spec.diffuse_ic else 0
    sc.keep_ic_gas_density = 1 if spec.keep_ic_gas_density else 0
    if spec.rho_ref is not None:
        sc.rho_ref[0], sc.rho_ref[1] = spec.rho_ref
    h = ctypes.c_void_p()
    rc = lib.dg_build_tree(ctypes.byref(sc), ctypes.byref(h))
    if rc != DG_OK:
        raise DgError(rc, lib.dg_build_last_error().decode())
    try:
        n = ctypes.c_longlong(0)
        lib.dg_tree_nodes(h, ctypes.byref(n))
        n = n.value
        C, NF = sh.C, sh.NF
        parent = np.zeros(n, np.int32)
        children = np.zeros((n, C), np.int32)
        level = np.zeros(n, np.int32)
        flags = np.zeros(n, np.uint32)
        bc = np.zeros((n, NF), np.int32)
        center = np.zeros((n, D), np.float64)
        p = np.zeros((n, E), np.float64)
        ip, up, dp = ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(_D)
        rc = lib.dg_tree_copy(h, parent.ctypes.data_as(ip), children.ctypes.data_as(ip), level.ctypes.data_as(ip),
                              flags.ctypes.data_as(up), bc.ctypes.data_as(ip), center.ctypes.data_as(dp),
                              p.ctypes.data_as(dp))
        if rc != DG_OK:
            raise DgError(rc, "dg_tree_copy failed")
    finally:
        lib.dg_tree_free(h)
    marked = (bc == -2).any(axis=1)
    if marked.any():
        # object faces: the nearest object's condition with the surface normal there, as the host
        # builder assigns them (scene._ObjectBoundaries)
        walls = _ObjectBoundaries(spec, D, E)
        nodes = np.nonzero(marked)[0]
        ids = walls.nearest(center[nodes], bcs)
        rows = bc[nodes]
        rows[rows == -2] = np.repeat(ids, (rows == -2).sum(axis=1))
        bc[nodes] = rows
    return Tree(shape=sh, parent=parent, children=children, level=level, flags=flags, bc=bc, center=center, p=p,
                bcs=bcs)
