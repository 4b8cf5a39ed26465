"""Initial tree builder for analytic scenes (host side).

Restates DACTI's ``Scene<M>::init_domain`` (scene/scene.cpp:369-431) for cases whose geometry is
analytic (spheres/circles instead of libigl meshes):

- the level-by-level loop of signed distances (scene.cpp:47-91), boundary tagging (:94-147),
  split detection (:150-216) and splitting (:219-245);
- leaves outside the active box become inactive and active leaves get the initial condition
  ``x2p(center)`` (:403-423);
- multiphase cases initialise the volume fraction near droplets (:343-365), optionally smeared
  with ``alpha = 0.5 (1 - tanh(sd / h))``, h = side_length / 2^max_level.

Child centres are computed exactly as ``Domain::split`` does (integrator/domain.hpp:206),
``parent.center + (0.25 * parent.size) * quadrant(i)``, so every centre is bit-identical to the
reference's. Cell sizes halve exactly per level from ``side_length``.

Without geometry objects the reference never assigns ``is_active`` before its final
"no objects -> every leaf active" pass (scene.cpp:389-398) and compares uninitialised flags while
tagging boundaries; here every node inside the root is active and only domain faces get
boundaries, which is what that pass intends.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np

from .models import (
    BcType,
    F_ACTIVE,
    F_CAN_SPLIT,
    F_CAN_UNSPLIT,
    F_IS_BOUNDARY,
    F_LEAF,
    F_SHOULD_SPLIT,
    ModelShape,
)


@dataclass
class BoundarySpec:
    """One Boundary<M> value (integrator/boundary.hpp:34-69)."""

    type: BcType
    p_in: Optional[Sequence[float]] = None
    normal: Optional[Sequence[float]] = None
    fade_in: float = 0.0


@dataclass
class SphereObject:
    """Analytic geometry object: signed distance |x - c| - r (negative inside)."""

    center: Sequence[float]
    radius: float
    type: str = "droplet"  # droplet | bubble | solid
    bc: Optional[BoundarySpec] = None

    def signed_distance(self, x: np.ndarray) -> np.ndarray:
        c = np.asarray(self.center, dtype=np.float64)[: x.shape[1]]
        return np.sqrt(((x - c) ** 2).sum(axis=1)) - self.radius


@dataclass
class EllipseObject:
    """Ellipse/ellipsoid with semi-axes `axes`, turned by `angle_deg` about z (2D), centred at `center`;
    signed distance approximated by (|y/a| - 1) * min(a) in the body frame y (exact on a circle), which
    is all the initial refinement and volume fraction need."""

    center: Sequence[float]
    axes: Sequence[float]
    type: str = "droplet"
    bc: Optional[BoundarySpec] = None
    angle_deg: float = 0.0

    def signed_distance(self, x: np.ndarray) -> np.ndarray:
        D = x.shape[1]
        c = np.asarray(self.center, dtype=np.float64)[:D]
        a = np.asarray(self.axes, dtype=np.float64)[:D]
        y = x - c
        if self.angle_deg != 0.0:
            if D != 2:
                raise NotImplementedError("rotated ellipsoids are supported in 2D only")
            th = self.angle_deg * math.pi / 180.0
            cs, sn = math.cos(th), math.sin(th)
            # body frame: R^T (x - c) with R the rotation by +angle about z
            y = np.stack([cs * y[:, 0] + sn * y[:, 1], -sn * y[:, 0] + cs * y[:, 1]], axis=1)
        return (np.sqrt(((y / a) ** 2).sum(axis=1)) - 1.0) * a.min()


@dataclass
class PolygonObject:
    """Closed 2D polygon (vertices in order, either orientation): exact signed distance, negative
    inside (even-odd rule)."""

    vertices: Sequence[Sequence[float]]
    type: str = "droplet"
    bc: Optional[BoundarySpec] = None

    def signed_distance(self, x: np.ndarray) -> np.ndarray:
        if x.shape[1] != 2:
            raise NotImplementedError("polygon objects are 2D")
        v = np.asarray(self.vertices, np.float64)
        w = np.roll(v, -1, axis=0)
        dist = np.full(x.shape[0], np.inf)
        inside = np.zeros(x.shape[0], bool)
        for a, b in zip(v, w):
            ab = b - a
            t = np.clip(((x - a) @ ab) / (ab @ ab), 0.0, 1.0)
            dist = np.minimum(dist, np.sqrt(((x - (a + t[:, None] * ab)) ** 2).sum(axis=1)))
            crosses = (a[1] > x[:, 1]) != (b[1] > x[:, 1])
            with np.errstate(divide="ignore", invalid="ignore"):
                xc = a[0] + (x[:, 1] - a[1]) * ab[0] / ab[1]
            inside ^= crosses & (x[:, 0] < xc)
        return np.where(inside, -dist, dist)


@dataclass
class RefineZone:
    """Refinement zone (config/config.hpp:77-86): cells whose centre, padded to 3D with zeros, lies
    strictly inside the box (x0, x1) may refine up to `level`."""

    x0: Sequence[float]
    x1: Sequence[float]
    level: int

    def __post_init__(self):
        if len(self.x0) != 3 or len(self.x1) != 3:
            raise ValueError("refinement zone corners are 3D points (vec3_t), also in 1D and 2D cases")

    def contains(self, ctr: np.ndarray) -> np.ndarray:
        x = np.zeros((ctr.shape[0], 3))
        x[:, : ctr.shape[1]] = ctr
        return np.all((x < np.asarray(self.x1, np.float64)) & (x > np.asarray(self.x0, np.float64)), axis=1)


@dataclass
class SceneSpec:
    shape: ModelShape
    active_size: Sequence[float]
    min_level: int
    max_level: int
    x2p: Callable[[np.ndarray], np.ndarray]  # (n, D) centres -> (n, E) primitives
    domain_bc: Sequence[Optional[tuple]]  # per dim: None (periodic) or (BoundarySpec neg, BoundarySpec pos)
    max_level_geom: Optional[int] = None
    refinement_radius: float = 2.0
    jump: Optional[tuple] = None  # (axis, location): refine around an initial jump (scene.cpp:193-200)
    objects: Sequence[SphereObject] = field(default_factory=list)
    zones: Sequence[RefineZone] = field(default_factory=list)
    diffuse_ic: bool = False
    rho_ref: Optional[Sequence[float]] = None  # multiphase phase densities (model/multi.hpp:479-483)
    # init_interface sets the gas density to rho_ref[1] (scene.cpp:362); True keeps a gas density the
    # initial condition already set (a shocked gas region) instead
    keep_ic_gas_density: bool = True

    @property
    def side_length(self) -> float:
        return float(max(self.active_size))

    @property
    def periodic(self) -> list:
        return [bc is None for bc in self.domain_bc]


@dataclass
class Tree:
    """Flat node arrays; slot 0 is the null node, slot 1 the root (integrator/domain.hpp:61-62)."""

    shape: ModelShape
    parent: np.ndarray
    children: np.ndarray  # (n, C)
    level: np.ndarray
    flags: np.ndarray  # uint32 F_* bits
    bc: np.ndarray  # (n, 2D) index into bcs or -1
    center: np.ndarray  # (n, D)
    p: np.ndarray  # (n, E)
    bcs: list

    @property
    def n_nodes(self) -> int:
        return int(self.parent.shape[0])

    def leaf_mask(self, active_only: bool = True) -> np.ndarray:
        m = (self.flags & F_LEAF) != 0
        if active_only:
            m &= (self.flags & F_ACTIVE) != 0
        m[0] = False
        return m


class _Grow:
    def __init__(self, shape: ModelShape, cap: int):
        D, E, C, NF = shape.dims, shape.E, shape.C, shape.NF
        self.n = 0
        self.parent = np.zeros(cap, np.int32)
        self.children = np.zeros((cap, C), np.int32)
        self.level = np.zeros(cap, np.int32)
        self.flags = np.zeros(cap, np.uint32)
        self.bc = np.full((cap, NF), -1, np.int32)
        self.center = np.zeros((cap, D), np.float64)
        self.size = np.zeros(cap, np.float64)
        self.p = np.zeros((cap, E), np.float64)
        self.sd = np.full(cap, np.finfo(np.float64).max)
        self.mesh = np.zeros(cap, np.int32)

    def reserve(self, extra: int) -> None:
        need = self.n + extra
        cap = self.parent.shape[0]
        if need <= cap:
            return
        new = max(need, 2 * cap)
        for name in ("parent", "children", "level", "flags", "bc", "center", "size", "p", "sd", "mesh"):
            a = getattr(self, name)
            b = np.empty((new,) + a.shape[1:], a.dtype)
            b[: a.shape[0]] = a
            if name == "bc":
                b[a.shape[0]:] = -1
            elif name == "sd":
                b[a.shape[0]:] = np.finfo(np.float64).max
            else:
                b[a.shape[0]:] = 0
            setattr(self, name, b)


def _quadrants(D: int) -> np.ndarray:
    """vec::quadrant(i) (core/linalg.hpp:67-80): +1 where bit d of i is set, else -1."""
    C = 1 << D
    q = np.empty((C, D), np.float64)
    for i in range(C):
        for d in range(D):
            q[i, d] = 1.0 if (i >> d) & 1 else -1.0
    return q


def build_tree(spec: SceneSpec) -> Tree:
    shape = spec.shape
    D, E, C = shape.dims, shape.E, shape.C
    side = spec.side_length
    act = np.asarray(spec.active_size, np.float64)[:D]
    if any(o.type == "solid" for o in spec.objects):
        raise NotImplementedError("solid geometry objects (object boundary tagging) are not supported yet")
    max_level_geom = spec.max_level if spec.max_level_geom is None else spec.max_level_geom

    # Boundary table: domain boundaries first, one entry per (dim, dir).
    bcs: list = []
    domain_bc_id = np.full((D, 2), -1, np.int32)
    for d in range(D):
        pair = spec.domain_bc[d]
        if pair is None:
            continue
        for side_dir in range(2):
            b = pair[side_dir]
            normal = [0.0] * D
            if b.type in (BcType.FREESLIP, BcType.NOSLIP):
                normal[d] = -(2.0 * side_dir - 1.0)  # scene.cpp:108 passes -unit(dim)*(2dir-1)
            domain_bc_id[d, side_dir] = len(bcs)
            bcs.append(
                BoundarySpec(b.type, list(b.p_in) if b.p_in is not None else [0.0] * E, normal, b.fade_in)
            )

    g = _Grow(shape, 1024)
    g.reserve(2)
    g.n = 2
    g.level[0] = -1
    g.parent[1] = 0
    g.level[1] = 0
    g.size[1] = side
    g.flags[1] = F_LEAF | F_ACTIVE | F_CAN_SPLIT
    quad = _quadrants(D)
    g.sd[0] = -1.0
    g.sd[1] = 0.0

    frontier = np.array([1], np.int64)
    while frontier.size:
        ctr = g.center[frontier]
        size = g.size[frontier]
        lvl = g.level[frontier]
        fl = g.flags[frontier]

        # compute_signed_distances (scene.cpp:47-91): minimum over objects.
        g.sd[frontier] = np.finfo(np.float64).max
        g.mesh[frontier] = 0
        for mi, obj in enumerate(spec.objects):
            dist = obj.signed_distance(ctr)
            closer = dist < g.sd[frontier]
            g.mesh[frontier[closer]] = mi
            g.sd[frontier[closer]] = dist[closer]
        sd = g.sd[frontier]

        # compute_node_boundaries (scene.cpp:94-147), domain faces only.
        g.bc[frontier] = -1
        for d in range(D):
            for side_dir in range(2):
                s = 2.0 * side_dir - 1.0
                ncen = ctr[:, d] + s * size
                if domain_bc_id[d, side_dir] >= 0:
                    out = ncen * s > act[d] / 2.0
                    g.bc[frontier[out], 2 * d + side_dir] = domain_bc_id[d, side_dir]

        # detect_splits (scene.cpp:150-216), in the reference's order of assignments.
        split = np.zeros(frontier.size, bool)
        cu = (fl & F_CAN_UNSPLIT) != 0
        below = lvl < spec.min_level
        split |= below
        cu[below] = False
        if spec.objects:
            near = np.abs(sd) < size * spec.refinement_radius
            solid = np.array([spec.objects[m].type == "solid" for m in g.mesh[frontier]], bool)
            m1 = near & solid & (lvl < max_level_geom)
            split |= m1
            cu[m1] = False
            m2 = near & ~solid & (lvl < spec.max_level)
            split |= m2
            cu[m2] = True
        for d in range(D):
            for side_dir in range(2):
                bid = g.bc[frontier, 2 * d + side_dir]
                has = bid >= 0
                if not has.any():
                    continue
                is_r = np.array([b >= 0 and bcs[b].type == BcType.INFLOW_R for b in bid], bool)
                m3 = is_r & (lvl < spec.max_level)
                split |= m3
                cu[m3] = True
        if spec.jump is not None:
            axis, loc = spec.jump
            m4 = (np.abs(ctr[:, axis] - loc) < size) & (lvl < spec.max_level)
            split |= m4
            cu[m4] = True
        for z in spec.zones:
            split |= z.contains(ctr) & (lvl < z.level)
        fl = np.where(cu, fl | F_CAN_UNSPLIT, fl & ~np.uint32(F_CAN_UNSPLIT)).astype(np.uint32)
        g.flags[frontier] = fl

        # split_detected_nodes (scene.cpp:219-245) with Domain::split (integrator/domain.hpp:192-247).
        parents = frontier[split & ((fl & F_LEAF) != 0)]
        npar = parents.size
        if npar == 0:
            break
        g.reserve(npar * C)
        first = g.n
        kids = first + np.arange(npar * C).reshape(npar, C)
        g.n += npar * C
        pc = g.center[parents]
        psz = g.size[parents]
        q = 0.25 * psz  # 0.25 * parent.size, then * quadrant(i)
        for i in range(C):
            k = kids[:, i]
            g.parent[k] = parents
            g.level[k] = g.level[parents] + 1
            g.center[k] = pc + q[:, None] * quad[i][None, :]
            g.size[k] = 0.5 * psz
            g.flags[k] = F_LEAF | F_ACTIVE | F_CAN_SPLIT | (g.flags[parents] & F_CAN_UNSPLIT)
        g.children[parents] = kids
        g.flags[parents] &= ~np.uint32(F_LEAF | F_SHOULD_SPLIT)
        frontier = kids.reshape(-1)

    n = g.n
    flags = g.flags[:n].copy()
    center = g.center[:n]
    # Cells whose centre lies outside the active box are inactive (scene.cpp:407-411).
    outside = np.zeros(n, bool)
    for d in range(D):
        outside |= (center[:, d] > 0.5 * act[d]) | (center[:, d] < -0.5 * act[d])
    outside[0] = False
    flags[outside] &= ~np.uint32(F_ACTIVE)
    flags[0] = 0
    p = np.zeros((n, E), np.float64)
    leaf = ((flags & F_LEAF) != 0) & ((flags & F_ACTIVE) != 0)
    leaf[0] = False
    idx = np.nonzero(leaf)[0]
    p[idx] = spec.x2p(center[idx])
    if shape.model == 2 and D > 1 and spec.objects:
        _init_interface(spec, g, idx, center, p)
    is_boundary = np.zeros(n, bool)
    return Tree(
        shape=shape,
        parent=g.parent[:n].copy(),
        children=g.children[:n].copy(),
        level=g.level[:n].copy(),
        flags=np.where(is_boundary, flags | F_IS_BOUNDARY, flags).astype(np.uint32),
        bc=g.bc[:n].copy(),
        center=center.copy(),
        p=p,
        bcs=bcs,
    )


def _init_interface(spec: SceneSpec, g: _Grow, idx: np.ndarray, center: np.ndarray, p: np.ndarray) -> None:
    """Scene::init_interface (scene/scene.cpp:343-365) with an optional tanh smear.

    The second phase density keeps the initial-condition value of ``p[1] / (1 - alpha_ic)`` where
    the IC already set one (a shocked air region), instead of resetting it to the reference
    density everywhere.
    """
    shape = spec.shape
    rho1, rho2 = spec.rho_ref
    sd = g.sd[idx].copy()
    kind = [spec.objects[m].type for m in g.mesh[idx]]
    alpha = np.zeros(idx.size)
    size = g.size[idx]
    h = spec.side_length / (1 << spec.max_level)
    for j, t in enumerate(kind):
        if t == "droplet":
            alpha[j] = 1.0 if sd[j] < 0 else 0.0
        elif t == "bubble":
            alpha[j] = 1.0 if sd[j] > 0 else 0.0
            sd[j] = -sd[j]
        else:
            alpha[j] = np.nan
    if spec.diffuse_ic:
        sm = np.abs(sd) < size * spec.refinement_radius
        alpha = np.where(sm & ~np.isnan(alpha), 0.5 * (1.0 - np.tanh(sd / h)), alpha)
    keep = np.isnan(alpha)
    ia = shape.ia
    if spec.keep_ic_gas_density:
        air = p[idx, 1] / np.where(p[idx, ia] < 1.0, 1.0 - p[idx, ia], 1.0)
        air = np.where(air > 0, air, rho2)
    else:
        air = np.full(idx.size, float(rho2))
    new = p[idx].copy()
    new[:, 0] = rho1 * alpha
    new[:, 1] = air * (1.0 - alpha)
    new[:, ia] = alpha
    p[idx] = np.where(keep[:, None], p[idx], new)
