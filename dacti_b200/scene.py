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

    def surface_normal(self, x: np.ndarray) -> np.ndarray:
        """Unit normal of the surface at the point nearest to each x."""
        c = np.asarray(self.center, dtype=np.float64)[: x.shape[1]]
        return _unit(x - c)

    def segment_hits(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        """Whether the segment a-b meets the surface."""
        c = np.asarray(self.center, dtype=np.float64)[: a.shape[1]]
        return _hits_unit_sphere((a - c) / self.radius, (b - c) / self.radius)

    def outline(self, n: int) -> np.ndarray:
        """n points of the 2D circle, counter-clockwise."""
        t = 2.0 * math.pi * np.arange(n) / n
        c = np.asarray(self.center, dtype=np.float64)[:2]
        return c + self.radius * np.stack([np.cos(t), np.sin(t)], axis=1)


def _unit(v: np.ndarray) -> np.ndarray:
    n = np.sqrt((v ** 2).sum(axis=1, keepdims=True))
    out = np.zeros_like(v)
    out[:, 0] = 1.0
    return np.where(n > 0, v / np.where(n > 0, n, 1.0), out)


def _hits_unit_sphere(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Segment a-b meets the unit sphere: its nearest point to the origin is inside or on it and its
    farthest point (an end) is outside or on it."""
    ab = b - a
    den = (ab ** 2).sum(axis=1)
    t = np.clip(-(a * ab).sum(axis=1) / np.where(den > 0, den, 1.0), 0.0, 1.0)
    near = a + t[:, None] * ab
    dmin = (near ** 2).sum(axis=1)
    dmax = np.maximum((a ** 2).sum(axis=1), (b ** 2).sum(axis=1))
    return (dmin <= 1.0) & (dmax >= 1.0)


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

    def _frame(self, x: np.ndarray):
        D = x.shape[1]
        c = np.asarray(self.center, dtype=np.float64)[:D]
        y = x - c
        th = self.angle_deg * math.pi / 180.0
        cs, sn = math.cos(th), math.sin(th)
        if D == 2 and self.angle_deg != 0.0:
            y = np.stack([cs * y[:, 0] + sn * y[:, 1], -sn * y[:, 0] + cs * y[:, 1]], axis=1)
        return y, np.asarray(self.axes, dtype=np.float64)[:D], cs, sn

    def surface_normal(self, x: np.ndarray) -> np.ndarray:
        """Unit normal of the level set through each x (the gradient of |y/a|), a stand-in for the
        normal at the nearest surface point."""
        y, a, cs, sn = self._frame(x)
        g = y / a ** 2
        if x.shape[1] == 2 and self.angle_deg != 0.0:
            g = np.stack([cs * g[:, 0] - sn * g[:, 1], sn * g[:, 0] + cs * g[:, 1]], axis=1)
        return _unit(g)

    def segment_hits(self, a_pt: np.ndarray, b_pt: np.ndarray) -> np.ndarray:
        """Whether the segment meets the surface (an affine map takes the ellipse to the unit circle)."""
        ya, a, _, _ = self._frame(a_pt)
        yb, _, _, _ = self._frame(b_pt)
        return _hits_unit_sphere(ya / a, yb / a)

    def outline(self, n: int) -> np.ndarray:
        """n points of the 2D ellipse, counter-clockwise."""
        t = 2.0 * math.pi * np.arange(n) / n
        a = np.asarray(self.axes, dtype=np.float64)[:2]
        y = np.stack([a[0] * np.cos(t), a[1] * np.sin(t)], axis=1)
        th = self.angle_deg * math.pi / 180.0
        R = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]])
        return np.asarray(self.center, dtype=np.float64)[:2] + y @ R.T


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
            # elementwise products and sums (no fused dot product): the device builder rounds the same way
            t = np.clip(((x[:, 0] - a[0]) * ab[0] + (x[:, 1] - a[1]) * ab[1]) / (ab[0] * ab[0] + ab[1] * ab[1]), 0.0, 1.0)
            e0, e1 = x[:, 0] - (a[0] + t * ab[0]), x[:, 1] - (a[1] + t * ab[1])
            dist = np.minimum(dist, np.sqrt(e0 * e0 + e1 * e1))
            crosses = (a[1] > x[:, 1]) != (b[1] > x[:, 1])
            with np.errstate(divide="ignore", invalid="ignore"):
                xc = a[0] + (x[:, 1] - a[1]) * ab[0] / ab[1]
            inside ^= crosses & (x[:, 0] < xc)
        return np.where(inside, -dist, dist)

    def surface_normal(self, x: np.ndarray) -> np.ndarray:
        """Unit vector from the nearest boundary point to x (the edge normal where x lies on an edge)."""
        v = np.asarray(self.vertices, np.float64)
        w = np.roll(v, -1, axis=0)
        best = np.full(x.shape[0], np.inf)
        nrm = np.zeros_like(x)
        for a, b in zip(v, w):
            ab = b - a
            t = np.clip(((x - a) @ ab) / (ab @ ab), 0.0, 1.0)
            d = x - (a + t[:, None] * ab)
            dist = np.sqrt((d ** 2).sum(axis=1))
            edge_n = np.array([ab[1], -ab[0]]) / math.hypot(ab[0], ab[1])
            cand = np.where((dist > 0)[:, None], d / np.where(dist > 0, dist, 1.0)[:, None], edge_n[None, :])
            closer = dist < best
            best = np.where(closer, dist, best)
            nrm[closer] = cand[closer]
        return nrm

    def outline(self, n: int = 0) -> np.ndarray:
        """The vertices, counter-clockwise."""
        v = np.asarray(self.vertices, np.float64)
        area2 = (v[:, 0] * np.roll(v[:, 1], -1) - np.roll(v[:, 0], -1) * v[:, 1]).sum()
        return v if area2 > 0 else v[::-1].copy()

    def segment_hits(self, p: np.ndarray, q: np.ndarray) -> np.ndarray:
        """Whether the segment p-q meets any edge (touching counts)."""
        v = np.asarray(self.vertices, np.float64)
        w = np.roll(v, -1, axis=0)

        def cross(o, a, b):
            return (a[..., 0] - o[..., 0]) * (b[..., 1] - o[..., 1]) - (a[..., 1] - o[..., 1]) * (b[..., 0] - o[..., 0])

        hit = np.zeros(p.shape[0], bool)
        for a, b in zip(v, w):
            A, B = np.broadcast_to(a, p.shape), np.broadcast_to(b, p.shape)
            d1, d2 = cross(A, B, p), cross(A, B, q)
            d3, d4 = cross(p, q, A), cross(p, q, B)
            hit |= (np.sign(d1) * np.sign(d2) <= 0) & (np.sign(d3) * np.sign(d4) <= 0) & \
                (np.minimum(p[:, 0], q[:, 0]) <= max(a[0], b[0])) & (np.maximum(p[:, 0], q[:, 0]) >= min(a[0], b[0])) & \
                (np.minimum(p[:, 1], q[:, 1]) <= max(a[1], b[1])) & (np.maximum(p[:, 1], q[:, 1]) >= min(a[1], b[1]))
        return hit


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
    # the initial condition as data, for the device builder: ("uniform", p) or ("jump", axis, location,
    # p_neg, p_pos) with p_pos where x[axis] > location; must agree with x2p
    ic: Optional[tuple] = None

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
        self.isb = np.zeros(cap, bool)

    def reserve(self, extra: int) -> None:
        need = self.n + extra
        cap = self.parent.shape[0]
        if need <= cap:
            return
        new = max(need, 2 * cap)
        for name in ("parent", "children", "level", "flags", "bc", "center", "size", "p", "sd", "mesh", "isb"):
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


def _find(g: "_Grow", pts: np.ndarray, max_lv: np.ndarray, act: np.ndarray, periodic: Sequence[bool]) -> np.ndarray:
    """Domain::find (integrator/domain.hpp:65-82, :407-417) for many points: the node at level <=
    max_lv containing each point (periodic wrap into the active box; 0 outside a non-periodic side).
    The descent compares with node centres, which is the reference's scaled-coordinate descent."""
    pts = np.array(pts, np.float64, copy=True)
    D = pts.shape[1]
    ok = np.ones(pts.shape[0], bool)
    for d in range(D):
        lo, hi = pts[:, d] < -0.5 * act[d], pts[:, d] > 0.5 * act[d]
        if periodic[d]:
            pts[lo, d] += act[d]
            pts[hi, d] -= act[d]
        else:
            ok &= ~(lo | hi)
    idx = np.where(ok, 1, 0).astype(np.int64)
    while True:
        go = ok & ((g.flags[idx] & F_LEAF) == 0) & (g.level[idx] < max_lv)
        if not go.any():
            break
        ii = idx[go]
        bits = np.zeros(ii.size, np.int64)
        for d in range(D):
            bits |= (pts[go, d] > g.center[ii, d]).astype(np.int64) << d
        idx[go] = g.children[ii, bits]
    return idx


class _ObjectBoundaries:
    """Boundaries of objects with a boundary condition (solids): Scene::nearest_boundary and
    Scene::raycast (scene/scene.cpp:11-45) over analytic shapes. Each boundary face gets the condition
    of the nearest object with a condition and, as its normal, the surface normal there; entries with
    equal values share one slot of the boundary table."""

    def __init__(self, spec: "SceneSpec", D: int, E: int):
        self.spec, self.D, self.E = spec, D, E
        self.keys: dict = {}

    def nearest(self, x: np.ndarray, bcs: list) -> np.ndarray:
        best = np.full(x.shape[0], np.inf)
        which = np.full(x.shape[0], -1)
        for mi, o in enumerate(self.spec.objects):
            if o.bc is None:
                continue
            dist = np.abs(o.signed_distance(x))
            closer = dist < best
            best = np.where(closer, dist, best)
            which[closer] = mi
        ids = np.empty(x.shape[0], np.int32)
        for mi in np.unique(which):
            o = self.spec.objects[mi]
            sel = which == mi
            normals = o.surface_normal(x[sel])
            p_in = list(o.bc.p_in) if o.bc.p_in is not None else [0.0] * self.E
            out = []
            for nrm in normals:
                key = (int(o.bc.type), tuple(p_in), tuple(float(v) for v in nrm), float(o.bc.fade_in))
                if key not in self.keys:
                    if len(bcs) >= 32767:
                        raise ValueError("more than 32767 distinct boundary entries (16-bit face boundary ids)")
                    self.keys[key] = len(bcs)
                    bcs.append(BoundarySpec(o.bc.type, p_in, list(key[2]), o.bc.fade_in))
                out.append(self.keys[key])
            ids[sel] = out
        return ids

    def raycast(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        """The first object in order that the segment meets or that has no condition decides: a hit
        is a boundary, an object without a condition ends the search with no boundary."""
        hit = np.zeros(a.shape[0], bool)
        open_ = np.ones(a.shape[0], bool)
        for o in self.spec.objects:
            if o.bc is None:
                break
            h = o.segment_hits(a, b) & open_
            hit |= h
            open_ &= ~h
        return hit


def _split(g: "_Grow", parents: np.ndarray, quad: np.ndarray, copy_bc: bool) -> np.ndarray:
    """Domain::split (integrator/domain.hpp:192-247) of leaf `parents`; returns the children (P, C).
    With copy_bc, each child takes the parent's boundaries on the faces it shares with the parent."""
    C, D = quad.shape
    npar = parents.size
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
        g.bc[k] = -1
        if copy_bc:
            for d in range(D):
                for side_dir in range(2):
                    if ((i >> d) & 1) == side_dir:
                        g.bc[k, 2 * d + side_dir] = g.bc[parents, 2 * d + side_dir]
    g.children[parents] = kids
    g.flags[parents] &= ~np.uint32(F_LEAF | F_SHOULD_SPLIT)
    return kids


def _neighbour_centres(ctr: np.ndarray, size: np.ndarray, d: int, side_dir: int) -> np.ndarray:
    ncen = ctr.copy()
    ncen[:, d] += (2.0 * side_dir - 1.0) * size
    return ncen


def _is_active(g: "_Grow", idx: np.ndarray) -> np.ndarray:
    return (idx != 0) & ((g.flags[idx] & F_ACTIVE) != 0)


def _object_faces(g, walls, bcs, nodes, act, periodic, D):
    """The object-boundary test of compute_node_boundaries (scene.cpp:112-127) for the faces without a
    boundary yet: a face whose same-level neighbour differs in activity, or whose centre-to-centre
    segment meets an object, gets the nearest object's condition. Returns the (nodes, 2D) hit mask."""
    ctr, size, lvl = g.center[nodes], g.size[nodes], g.level[nodes]
    me = _is_active(g, nodes)
    hits = np.zeros((nodes.size, 2 * D), bool)
    for d in range(D):
        for side_dir in range(2):
            f = 2 * d + side_dir
            todo = g.bc[nodes, f] < 0
            if not todo.any():
                continue
            ncen = _neighbour_centres(ctr[todo], size[todo], d, side_dir)
            nb = _find(g, ncen, lvl[todo], act, periodic)
            hit = (_is_active(g, nb) != me[todo]) | walls.raycast(ctr[todo], ncen)
            sel = np.nonzero(todo)[0][hit]
            if sel.size:
                g.bc[nodes[sel], f] = walls.nearest(ctr[sel], bcs)
            hits[sel, f] = True
    return hits


def _fix_boundary(g, walls, bcs, quad, act, periodic, D):
    """Scene::fix_boundary (scene/scene.cpp:249-337): split active leaves coarser than an inactive
    neighbouring leaf until every inactive leaf meets same-level cells, recompute the boundaries of
    the new leaves (the reference skips its domain-face branch there, so a new leaf on the domain edge
    takes the nearest object's condition), then drop one-sided boundaries: a boundary of an active
    leaf whose neighbour has none on the opposite face. The splitting and the dropping run to their
    fixed points rather than in the reference's node order."""
    new_leaves: set = set()
    while True:
        idx = np.arange(1, g.n)
        inact = idx[((g.flags[1:g.n] & F_LEAF) != 0) & ((g.flags[1:g.n] & F_ACTIVE) == 0)]
        targets = []
        for d in range(D):
            for side_dir in range(2):
                ncen = _neighbour_centres(g.center[inact], g.size[inact], d, side_dir)
                nb = _find(g, ncen, g.level[inact], act, periodic)
                m = _is_active(g, nb) & (g.level[nb] < g.level[inact])
                targets.append(nb[m])
        t = np.unique(np.concatenate(targets)) if targets else np.zeros(0, np.int64)
        if t.size == 0:
            break
        kids = _split(g, t, quad, copy_bc=True)
        new_leaves.difference_update(t.tolist())
        new_leaves.update(kids.reshape(-1).tolist())
    if new_leaves:
        nl = np.array(sorted(new_leaves), np.int64)
        g.bc[nl] = -1
        _object_faces(g, walls, bcs, nl, act, periodic, D)
    while True:
        idx = np.arange(1, g.n)
        al = idx[((g.flags[1:g.n] & F_LEAF) != 0) & ((g.flags[1:g.n] & F_ACTIVE) != 0)]
        drop = []
        for d in range(D):
            for side_dir in range(2):
                f = 2 * d + side_dir
                has = al[g.bc[al, f] >= 0]
                ncen = _neighbour_centres(g.center[has], g.size[has], d, side_dir)
                nb = _find(g, ncen, g.level[has], act, periodic)
                rm = (nb != 0) & (g.bc[nb, 2 * d + 1 - side_dir] < 0)
                drop.append((has[rm], f))
        changed = False
        for nodes, f in drop:
            if nodes.size:
                g.bc[nodes, f] = -1
                changed = True
        if not changed:
            break


def build_tree(spec: SceneSpec) -> Tree:
    shape = spec.shape
    D, E, C = shape.dims, shape.E, shape.C
    side = spec.side_length
    act = np.asarray(spec.active_size, np.float64)[:D]
    periodic = spec.periodic
    walls = _ObjectBoundaries(spec, D, E) if any(o.bc is not None for o in spec.objects) else None
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
        if spec.objects:
            # scene.cpp:76-82: inside an object with a boundary condition is inactive
            has_bc = np.array([spec.objects[m].bc is not None for m in g.mesh[frontier]], bool)
            fl = np.where((sd < 0.0) & has_bc, fl & ~np.uint32(F_ACTIVE), fl | F_ACTIVE).astype(np.uint32)
            g.flags[frontier] = fl

        # compute_node_boundaries (scene.cpp:94-147): domain faces, then object faces.
        g.bc[frontier] = -1
        for d in range(D):
            for side_dir in range(2):
                s = 2.0 * side_dir - 1.0
                ncen = ctr[:, d] + s * size
                if domain_bc_id[d, side_dir] >= 0:
                    out = ncen * s > act[d] / 2.0
                    g.bc[frontier[out], 2 * d + side_dir] = domain_bc_id[d, side_dir]
        objb = np.zeros(frontier.size, bool)
        if walls is not None:
            # neighbours' activity as it stands after the distance pass (the reference reads it while
            # other threads clear it)
            objb = _object_faces(g, walls, bcs, frontier, act, periodic, D).any(axis=1)
            no_open = ~(g.bc[frontier] < 0).any(axis=1)
            fl = np.where(no_open, fl & ~np.uint32(F_ACTIVE), fl).astype(np.uint32)
            g.isb[frontier[objb]] = True

        # detect_splits (scene.cpp:150-216), in the reference's order of assignments.
        split = np.zeros(frontier.size, bool)
        cu = (fl & F_CAN_UNSPLIT) != 0
        cu[objb] = False
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
        if parents.size == 0:
            break
        frontier = _split(g, parents, quad, copy_bc=False).reshape(-1)

    if walls is not None:
        for _ in range(10):  # init_domain calls fix_boundary ten times (scene.cpp:401-402)
            _fix_boundary(g, walls, bcs, quad, act, periodic, D)
        # leaves added by fix_boundary get distances for the interface initialisation
        nodes = np.arange(1, g.n)
        fresh = nodes[g.sd[nodes] == np.finfo(np.float64).max]
        for mi, obj in enumerate(spec.objects):
            if fresh.size == 0:
                break
            dist = obj.signed_distance(g.center[fresh])
            closer = dist < g.sd[fresh]
            g.mesh[fresh[closer]] = mi
            g.sd[fresh[closer]] = dist[closer]

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
    is_boundary = g.isb[:n].copy()
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
