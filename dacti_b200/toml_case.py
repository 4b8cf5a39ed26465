"""DACTI TOML case files (config/config.cpp:10-243, config/config.hpp:11-118) loaded into a `Case`.

`load_toml_case(path)` reads the same keys as `Config<M>::load_config` with the same defaults, type
rules and error behaviour, and builds the initial tree with the analytic scene builder:

- [scene] name, domain_size (side_length = max); [run] print_interval, end_time, signal_time (-1),
  steady_tol (-1); [integrator] max_cfl, max_dt (print_interval), min/max_refinement_level,
  max_refinement_level_geom (max level), refinement_radius (2), error_threshold, error_weights (ones);
- [model.reference_values] through the model's `dict` (model/euler.hpp:288-323,
  model/navier_stokes.hpp:120-134, model/multi.hpp:474-548), including the Navier-Stokes viscosity
  mu = rho |vel| L / Re and conductivity mu cp / Pr, and the multiphase We/Re/Oh/sigma/mu_ratio and
  fluid_1/fluid_2 constants;
- [initial_condition] uniform (reference / fixed) and jump; [boundary_conditions.X|Y|Z] periodic or
  neg/pos of noslip, freeslip, inflow, inflow_r, outflow, zeroGradient (config.cpp:145-190);
- [[geometry]] built-in 2D shapes ellipse, circle, diamond, quadrilateral, triangle, line, naca_airfoil
  and Joukowski_airfoil (the airfoils as densely sampled polygons) with their
  transform (rotation about z, scaling, translation: x = R S y + t, object_mesh.cpp:92-94) as
  analytic signed distances instead of the sampled line meshes the reference builds;
- [[refinement_zone]] start, end, max_refinement_level, transform_like (translation and scaling).

Type rules of `get_entry` (config/util.hpp:16-103): scalars must be TOML floats (an integer such as
`p = 1` is an error), integers must be TOML integers, vectors must be float arrays of the exact length.
A missing required key raises ConfigError, the reference's runtime_error("Config Error").

Reproduced quirks of the reference parser:

- `diffuse_ic` is looked up under initial_condition.initial_condition (config.cpp:198-199) and so is
  never set from the file; `honour_diffuse_ic=True` reads it where the file puts it;
- uniform/"fixed" requires `fixed_value` but initialises with the reference state (config.cpp:208-210);
- a multiphase `Ma` velocity uses the sound speed with the default fluid constants, since
  fluid_1/fluid_2 are parsed after it (model/multi.hpp:491-499, :537-547);
- `transform_like` naming no geometry gives the identity transform (std::unordered_map::operator[]).

Objects with a boundary condition (solids) make the cells inside them inactive and give the faces
towards them the condition, with the shape's normal (scene/scene.cpp:47-147, :249-337).

Not supported, with a clear error: STL geometry files (`path`), airfoil and line shapes, built-in
shapes in 3D, and refinement zones with a rotated transform.
"""
from __future__ import annotations

import math
import os
import tomllib
from dataclasses import dataclass, field
from typing import Any, Callable, Optional

import numpy as np

from .casefile import Case, SolverParams
from .models import BcType, ModelId, ModelShape
from .scene import BoundarySpec, EllipseObject, PolygonObject, RefineZone, SceneSpec, build_tree

MODELS = {"euler": ModelId.EULER, "navier_stokes": ModelId.NAVIER_STOKES, "multi": ModelId.MULTI}
_MISSING = object()
NS_CP = 1005.0  # navier_stokes::cp (model/navier_stokes.hpp:27)


class ConfigError(RuntimeError):
    """A missing or mistyped entry, or an unknown type name (config/util.hpp:25-26 and
    config/config.cpp:189, :242)."""


@dataclass
class RunSettings:
    """The [run] keys the driver loop reads (driver/default_driver.hpp:77-217)."""

    name: str
    io_interval: float
    end_time: float
    signal_time: float
    convergence_tol: float


@dataclass
class TomlCase:
    case: Case
    spec: SceneSpec
    run: RunSettings
    model: str
    p_ref: np.ndarray
    vel_ref: np.ndarray
    rho_ref: Optional[tuple]
    ignored: list = field(default_factory=list)  # keys present in the file that the reference ignores
    objects: list = field(default_factory=list)  # the analytic geometry objects, for observers


def _at_path(table: dict, path: str):
    node: Any = table
    for part in path.split("."):
        if not isinstance(node, dict) or part not in node:
            return _MISSING
        node = node[part]
    return node


def _is_float(v) -> bool:
    return isinstance(v, float)


def _is_int(v) -> bool:
    return isinstance(v, int) and not isinstance(v, bool)


def get_entry(table: dict, path: str, kind: str, default=_MISSING, size: int = 0):
    """config::get_entry: kind is "float", "int", "uint", "str", "bool" or "vec" (a float array of
    `size` entries)."""
    v = _at_path(table, path)
    if v is _MISSING:
        if default is not _MISSING:
            return default
        raise ConfigError(f"Config: Couldn't find entry for {path}.")
    if kind == "vec":
        if not isinstance(v, list):
            raise ConfigError(f"Config: Type of {path} should be array")
        if len(v) != size:
            raise ConfigError(f"Config: Length of {path} should be {size}, but is {len(v)}")
        for i, x in enumerate(v):
            if not _is_float(x):
                raise ConfigError(f"Config: Type of {path}[{i}] should be floating point")
        return np.array(v, np.float64)
    if kind == "float":
        if not _is_float(v):
            raise ConfigError(f"Config: Type of {path} should be floating point")
        return float(v)
    if kind in ("int", "uint"):
        if not _is_int(v):
            raise ConfigError(f"Config: Type of {path} should be int")
        if kind == "uint" and v < 0:
            raise ConfigError(f"Config: {path} should be unsigned, but a value of {v} was specified")
        return int(v)
    if kind == "str":
        if not isinstance(v, str):
            raise ConfigError(f"Config: Type of {path} should be string")
        return v
    if kind == "bool":
        if not isinstance(v, bool):
            raise ConfigError(f"Config: Type of {path} should be boolean")
        return v
    raise ValueError(kind)


def _table(parent: dict, key: str, what: str) -> dict:
    t = parent.get(key) if isinstance(parent, dict) else None
    if not isinstance(t, dict):
        raise ConfigError(f"Config: missing table {what}")
    return t


def infer_model(doc: dict) -> str:
    """The reference picks the model at compile time (src/examples/*.cpp); a file without that choice
    is read as multiphase when reference_values.rho is an array, Navier-Stokes when it gives Re, Euler
    otherwise."""
    ref = _at_path(doc, "model.reference_values")
    if isinstance(ref, dict) and isinstance(ref.get("rho"), list):
        return "multi"
    if isinstance(ref, dict) and "Re" in ref:
        return "navier_stokes"
    return "euler"


# multi::gamma / multi::p0 (model/multi.hpp:367-387) at given fluid constants.
def _multi_gamma(a: float, g1: float, g2: float) -> float:
    if a < 1e-20:
        return g2
    if a > 1 - 1e-20:
        return g1
    return 1 + 1 / (a / (g1 - 1) + (1 - a) / (g2 - 1))


def _multi_p0(a: float, g1: float, g2: float, P1: float, P2: float) -> float:
    if a < 1e-20:
        return P2
    if a > 1 - 1e-20:
        return P1
    return (a * g1 * P1 / (g1 - 1) + (1 - a) * g2 * P2 / (g2 - 1)) / (1 + a / (g1 - 1) + (1 - a) / (g2 - 1))


def _velocity_from_angle(D: int, mag: float, angle_deg: float) -> np.ndarray:
    if D < 2:
        raise ConfigError("vel_magnt/Ma reference velocities need at least two dimensions")
    vel = np.zeros(D)
    th = angle_deg * math.pi / 180
    vel[0], vel[1] = mag * math.cos(th), mag * math.sin(th)
    return vel


def _model_dict(model: str, D: int, mdl: dict, prm: SolverParams):
    """M::dict: fills p_ref, vel_ref, rho_ref and the model constants in `prm`."""
    ref = _table(mdl, "reference_values", "model.reference_values")
    if model in ("euler", "navier_stokes"):
        rho = get_entry(ref, "rho", "float")
        prs = get_entry(ref, "p", "float")
        if "vel_magnt" in ref:  # model/euler.hpp:294-299
            vel = _velocity_from_angle(D, get_entry(ref, "vel_magnt", "float"),
                                       get_entry(ref, "vel_angle", "float", 0.0))
        elif "Ma" in ref:  # model/euler.hpp:300-314
            mag = get_entry(ref, "Ma", "float") * math.sqrt(1.4 * prs / rho)
            ang = get_entry(ref, "vel_angle", "float", 0.0) * math.pi / 180
            vel = np.zeros(D)
            if D == 2:
                vel[:] = mag * math.cos(ang), mag * math.sin(ang)
            elif D == 3:
                vel[:] = -mag * math.cos(ang), 0.0, mag * math.sin(ang)
            else:
                raise ConfigError("a Mach-number reference velocity needs two or three dimensions")
        else:
            vel = get_entry(ref, "vel", "vec", size=D)
        p_ref = np.concatenate([[rho], vel, [prs]])
        if model == "navier_stokes":  # model/navier_stokes.hpp:120-134
            Re = get_entry(ref, "Re", "float")
            L = get_entry(ref, "L", "float")
            prm.ns_mu = p_ref[0] * float(np.linalg.norm(vel)) * L / Re
            if "Pr" in ref:
                prm.ns_lambda = prm.ns_mu * NS_CP / get_entry(ref, "Pr", "float")
        return p_ref, vel, None
    # multi (model/multi.hpp:474-548)
    rho = get_entry(ref, "rho", "vec", size=2)
    prs = get_entry(ref, "p", "float")
    alpha = get_entry(ref, "alpha", "float")
    if "vel_magnt" in ref:
        vel = _velocity_from_angle(D, get_entry(ref, "vel_magnt", "float"), get_entry(ref, "vel_angle", "float", 0.0))
    elif "Ma" in ref:
        mach = get_entry(ref, "Ma", "float")
        ang = get_entry(ref, "vel_angle", "float", 0.0)
        ra = (rho[0] * alpha, rho[1] * (1 - alpha))
        # the fluid constants here are still the defaults: fluid_1/fluid_2 are read further down
        g = _multi_gamma(alpha, prm.gamma1, prm.gamma2)
        c = math.sqrt(g * (prs + _multi_p0(alpha, prm.gamma1, prm.gamma2, prm.P1, prm.P2)) / (ra[0] + ra[1]))
        vel = _velocity_from_angle(D, mach * c, ang)
    else:
        vel = get_entry(ref, "vel", "vec", size=D)
    p_ref = np.concatenate([[rho[0] * alpha, rho[1] * (1.0 - alpha)], vel, [prs, alpha]])
    L = get_entry(ref, "L", "float", 1.0)
    mu_ratio = get_entry(ref, "mu_ratio", "float", 1.0)
    We = None
    if "We" in ref:
        We = get_entry(ref, "We", "float")
        prm.sigma = 1.0 / We
    if "Re" in ref:
        Re = get_entry(ref, "Re", "float")
        if We is None:
            raise ConfigError("model.reference_values.Re needs We (the reference reads an unset We)")
        prm.mu1 = math.sqrt(rho[0] * prm.sigma * L) * math.sqrt(We) / Re
        prm.mu2 = prm.mu1 / mu_ratio
    if "Oh" in ref:
        Oh = get_entry(ref, "Oh", "float")
        prm.sigma = get_entry(ref, "sigma", "float")
        prm.mu1 = math.sqrt(rho[0] * prm.sigma * L) * Oh
        prm.mu2 = prm.mu1 / mu_ratio
    if "fluid_1" in mdl:
        f1 = _table(mdl, "fluid_1", "model.fluid_1")
        prm.P1 = get_entry(f1, "P0", "float", prm.P1)
        prm.gamma1 = get_entry(f1, "gamma", "float", prm.gamma1)
    if "fluid_2" in mdl:
        f2 = _table(mdl, "fluid_2", "model.fluid_2")
        prm.P2 = get_entry(f2, "P0", "float", prm.P2)
        prm.gamma2 = get_entry(f2, "gamma", "float", prm.gamma2)
    return p_ref, vel, (float(rho[0]), float(rho[1]))


def _boundary(tab: dict, shape: ModelShape, p_ref: np.ndarray) -> BoundarySpec:
    """Config::parse_boundary_condition (config/config.cpp:145-190)."""
    typ = get_entry(tab, "type", "str")
    E = shape.E
    if typ == "noslip":
        return BoundarySpec(BcType.NOSLIP)
    if typ == "freeslip":
        return BoundarySpec(BcType.FREESLIP)
    if typ == "inflow":
        return BoundarySpec(BcType.INFLOW, list(p_ref), None, get_entry(tab, "fade_in", "float", 0.0))
    if typ == "inflow_r":
        fade = get_entry(tab, "fade_in", "float", 0.0)
        return BoundarySpec(BcType.INFLOW_R, list(get_entry(tab, "value", "vec", size=E)), None, fade)
    if typ == "outflow":
        p = [0.0] * E
        p[shape.ip] = float(p_ref[shape.ip])
        return BoundarySpec(BcType.OUTFLOW, p)
    if typ == "zeroGradient":
        return BoundarySpec(BcType.ZERO_GRADIENT)
    raise ConfigError("illegal bc type")


def _initial_condition(ic: dict, shape: ModelShape, p_ref: np.ndarray, ignored: list, honour_diffuse: bool):
    """Config::parse_initial_condition (config/config.cpp:193-243): (x2p, jump, diffuse_ic)."""
    typ = get_entry(ic, "type", "str")
    diffuse = False
    if "diffuse_ic" in ic:
        if honour_diffuse:
            diffuse = get_entry(ic, "diffuse_ic", "bool")
        else:
            ignored.append("initial_condition.diffuse_ic")
    E = shape.E
    if typ == "uniform":
        value = get_entry(ic, "value", "str", "reference")
        if value in ("reference", "fixed"):
            if value == "fixed":
                get_entry(ic, "fixed_value", "vec", size=E)  # required, then unused
                ignored.append("initial_condition.fixed_value")
            ref = np.asarray(p_ref, np.float64)
            return (lambda c: np.tile(ref, (c.shape[0], 1))), None, diffuse
        raise ConfigError(f"Unknown uniform value type {value}")
    if typ == "jump":
        axis = get_entry(ic, "axis", "uint")
        loc = get_entry(ic, "location", "float")
        neg = get_entry(ic, "value_neg", "vec", size=E)
        pos = get_entry(ic, "value_pos", "vec", size=E)
        if axis >= shape.dims:
            raise ConfigError(f"initial_condition.axis {axis} is not a dimension of this case")
        return (lambda c: np.where((c[:, axis] > loc)[:, None], pos[None, :], neg[None, :])), (axis, loc), diffuse
    raise ConfigError(f"Unknown initial condition type {typ}")


@dataclass
class _Transform:
    rotation: np.ndarray
    scaling: np.ndarray
    translation: np.ndarray

    def identity(self) -> bool:
        return (not self.rotation.any()) and bool((self.scaling == 1.0).all()) and not self.translation.any()


def _naca4_outline(m: float, p: float, t: float, n: int = 400) -> np.ndarray:
    """NACA4Airfoil (scene/geometry.hpp:57-100) sampled as a polygon: the parameter x in [-1, 1] runs
    along the lower surface (x < 0) from the trailing edge to the leading edge and back along the upper
    one. The chord runs from -0.5 to 0.5, and the closed trailing edge uses the -0.1036 x^4 thickness
    term. Points are cosine-spaced in |x|, dense at both edges; the shared trailing-edge point appears
    once."""
    u = 0.5 * (1.0 - np.cos(np.linspace(0.0, math.pi, n // 2 + 1)))       # 0 .. 1

    def point(x, sgn):
        yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x * x + 0.2843 * x ** 3 - 0.1036 * x ** 4)
        front = x < p
        with np.errstate(divide="ignore", invalid="ignore"):
            yc = np.where(front, m * (2 * p * x - x * x) / (p * p), m * (1 - 2 * p + 2 * p * x - x * x) / ((1 - p) ** 2))
            dy = np.where(front, 2 * m * (p - x) / (p * p), 2 * m * (p - x) / ((1 - p) ** 2))
        th = np.arctan(dy)
        return np.stack([x - sgn * yt * np.sin(th) - 0.5, yc + sgn * yt * np.cos(th)], axis=1)

    lower = point(u[::-1], -1.0)[:-1]        # trailing edge .. just before the leading edge
    upper = point(u, 1.0)[:-1]               # leading edge .. just before the trailing edge
    return np.concatenate([lower, upper])


def _joukowski_outline(m: float, t: float, delta: float, n: int = 400) -> np.ndarray:
    """JoukowskiAirfoil (scene/geometry.hpp:102-160) sampled as a polygon. The unit circle around
    zeta0 = (-t/1.299, 2m) is mapped by the Karman-Trefftz transform with exponent 2 - delta/180, then
    shifted to the mid-chord and scaled to unit chord; theta runs over [0, 2 pi)."""
    xc, yc = -t / 1.299, 2.0 * m
    zeta0 = complex(xc, yc)
    beta = math.asin(yc)
    a = math.cos(beta) + xc
    k = 2.0 - delta / 180.0

    def tr(z):
        return 0.5 * k * a * ((z + a) ** k + (z - a) ** k) / ((z + a) ** k - (z - a) ** k)

    le = tr(np.exp(1j * (beta + math.pi)) + zeta0).real
    te = tr(np.exp(1j * (-beta)) + zeta0).real
    chord = te - le
    theta = np.linspace(0.0, 2.0 * math.pi, n, endpoint=False)
    with np.errstate(divide="ignore", invalid="ignore"):
        z = (tr(np.exp(1j * theta) + zeta0) - 0.5 * (le + te)) / chord
    z = z[np.isfinite(z)]
    return np.stack([z.real, z.imag], axis=1)


def _geometry(g: dict, D: int, bc: Optional[BoundarySpec]):
    """One [[geometry]] entry: (object, transform) for the supported built-in shapes."""
    name = g.get("name")
    if not isinstance(name, str):
        raise ConfigError("Config: geometry entries need a string name")
    typ = get_entry(g, "type", "str", "solid")
    t = _Transform(get_entry(g, "rotation", "vec", np.zeros(3), 3), get_entry(g, "scaling", "vec", np.ones(3), 3),
                   get_entry(g, "translation", "vec", np.zeros(3), 3))
    if "path" in g:
        raise NotImplementedError(f"geometry '{name}': STL geometry files need mesh signed distances, which this "
                                  "build does not have; use a built-in shape")
    if "shape" not in g:
        raise ConfigError("Undefined Geometry")
    if D != 2:
        raise NotImplementedError(f"geometry '{name}': built-in shapes are 2D curves (extruded in 3D by the "
                                  "reference); only 2D cases take them here")
    if t.rotation[0] != 0.0 or t.rotation[1] != 0.0:
        raise NotImplementedError(f"geometry '{name}': only rotations about z apply to a 2D shape")
    if (t.scaling[:2] <= 0).any():
        raise ConfigError(f"geometry '{name}': scaling must be positive")
    shape = get_entry(g, "shape", "str")
    c = t.translation[:2]
    th = t.rotation[2] * math.pi / 180
    R = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]])
    S = t.scaling[:2]
    if shape == "ellipse":
        axes = (get_entry(g, "a", "float") * S[0], get_entry(g, "b", "float") * S[1])
        return EllipseObject(tuple(c), axes, typ, bc, float(t.rotation[2])), t
    if shape == "circle":
        r = get_entry(g, "radius", "float")
        return EllipseObject(tuple(c), (r * S[0], r * S[1]), typ, bc, float(t.rotation[2])), t
    if shape in ("diamond", "quadrilateral", "triangle"):
        if shape == "diamond":
            a, b = get_entry(g, "width", "float"), get_entry(g, "height", "float")
            v = np.array([[0, b / 2], [a / 2, 0], [0, -b / 2], [-a / 2, 0]], np.float64)
        else:
            keys = ("v1", "v2", "v3", "v4") if shape == "quadrilateral" else ("v1", "v2", "v3")
            v = np.array([get_entry(g, k, "vec", size=2) for k in keys])
        world = (v * S[None, :]) @ R.T + c[None, :]
        return PolygonObject(world.tolist(), typ, bc), t
    if shape == "line":
        # geometry_data.hpp:75-93: a segment of `length` centred on the origin along x, else v1-v2; a
        # two-vertex polygon here: no cell lies inside it, and every face whose centre-to-centre
        # segment crosses it takes the object's condition, from both sides (a plate of no thickness)
        length = get_entry(g, "length", "float", 0.0)
        if length > 0.0:
            v = np.array([[-length / 2.0, 0.0], [length / 2.0, 0.0]])
        else:
            v = np.array([get_entry(g, "v1", "vec", size=2), get_entry(g, "v2", "vec", size=2)])
        world = (v * S[None, :]) @ R.T + c[None, :]
        return PolygonObject(world.tolist(), typ, bc), t
    if shape in ("naca_airfoil", "Joukowski_airfoil"):
        # geometry_data.hpp:57-73; sampled densely here, adaptively (then meshed) in the reference
        camber, thick = get_entry(g, "camber", "float"), get_entry(g, "thickness", "float")
        if shape == "naca_airfoil":
            v = _naca4_outline(camber, get_entry(g, "position", "float"), thick)
        else:
            v = _joukowski_outline(camber, thick, get_entry(g, "trailing_edge_angle", "float", 0.0))
        world = (v * S[None, :]) @ R.T + c[None, :]
        return PolygonObject(world.tolist(), typ, bc), t
    raise ConfigError("Unknown shape type")


def load_toml_case(path: str, model: Optional[str] = None, limiter: int = 0, honour_diffuse_ic: bool = False,
                   x2p: Optional[Callable[[np.ndarray], np.ndarray]] = None, builder: str = "host") -> TomlCase:
    """Reads a DACTI case file into an initial tree and solver parameters. `model` is "euler",
    "navier_stokes" or "multi" (the reference's compile-time choice; inferred from the file if None);
    `limiter` is the slope limiter id (the examples use minmod, 0); `x2p` replaces the initial condition
    for states TOML cannot express, as code that sets Config::ic.x2p does. `builder` picks the tree
    builder: "host" (numpy), "device" (dg_build_tree on the current GPU; droplet/bubble scenes only) or
    "auto" (the device where the scene allows it, else the host)."""
    with open(path, "rb") as f:
        doc = tomllib.load(f)
    model = model or infer_model(doc)
    if model not in MODELS:
        raise ValueError(f"model must be one of {sorted(MODELS)}")
    size = _at_path(doc, "scene.domain_size")
    D = len(size) if isinstance(size, list) else 0
    if D not in (1, 2, 3):
        raise ConfigError("Config: scene.domain_size must be an array of 1 to 3 floats")
    shape = ModelShape(MODELS[model], D)
    ignored: list = []

    name = get_entry(doc, "scene.name", "str")
    active = get_entry(doc, "scene.domain_size", "vec", size=D)
    side = float(active.max())
    io_interval = get_entry(doc, "run.print_interval", "float")
    end_time = get_entry(doc, "run.end_time", "float")
    signal_time = get_entry(doc, "run.signal_time", "float", -1.0)
    steady_tol = get_entry(doc, "run.steady_tol", "float", -1.0)
    max_cfl = get_entry(doc, "integrator.max_cfl", "float")
    max_dt = get_entry(doc, "integrator.max_dt", "float", io_interval)
    min_level = get_entry(doc, "integrator.min_refinement_level", "int")
    max_level = get_entry(doc, "integrator.max_refinement_level", "int")
    max_level_geom = get_entry(doc, "integrator.max_refinement_level_geom", "int", max_level)
    radius = get_entry(doc, "integrator.refinement_radius", "float", 2.0)
    thresholds = get_entry(doc, "integrator.error_threshold", "vec", size=2)
    weights = get_entry(doc, "integrator.error_weights", "vec", np.ones(shape.E), shape.E)
    if "visualize_mesh" in doc.get("scene", {}):
        ignored.append("scene.visualize_mesh")

    prm = SolverParams(side_length=side, active_size=tuple(active), periodic=[False] * D, max_cfl=max_cfl,
                       max_dt=max_dt, error_threshold=tuple(thresholds), max_level=max_level, min_level=min_level,
                       weights=tuple(weights), limiter=limiter)
    mdl = doc.get("model")
    if not isinstance(mdl, dict):
        raise ConfigError("Config: missing table model")
    p_ref, vel_ref, rho_ref = _model_dict(model, D, mdl, prm)

    ic = doc.get("initial_condition")
    if not isinstance(ic, dict):
        raise ConfigError("Config: missing table initial_condition")
    ic_x2p, jump, diffuse = _initial_condition(ic, shape, p_ref, ignored, honour_diffuse_ic)

    bcs_doc = doc.get("boundary_conditions", {})
    domain_bc = []
    for d, dn in enumerate("XYZ"[:D]):
        tab = bcs_doc.get(dn, {}) if isinstance(bcs_doc, dict) else {}
        typ = tab.get("type") if isinstance(tab, dict) else None
        if isinstance(typ, str):
            if typ != "periodic":
                raise ConfigError(f"boundary_conditions.{dn}.type '{typ}': only 'periodic' may stand there "
                                  "(other conditions go under neg/pos)")
            domain_bc.append(None)
            continue
        neg, pos = tab.get("neg") if isinstance(tab, dict) else None, tab.get("pos") if isinstance(tab, dict) else None
        if not isinstance(neg, dict) or not isinstance(pos, dict):
            raise ConfigError(f"Config: boundary_conditions.{dn} needs neg and pos tables")
        domain_bc.append((_boundary(neg, shape, p_ref), _boundary(pos, shape, p_ref)))
    prm.periodic = [b is None for b in domain_bc]

    objects, transforms = [], {}
    for g in doc.get("geometry", []):
        gname = g.get("name")
        btab = bcs_doc.get(gname) if isinstance(bcs_doc, dict) and isinstance(gname, str) else None
        if get_entry(g, "type", "str", "solid") == "solid" and btab is None:
            raise ConfigError(f"Must define boundary condition for solid geometry '{gname}'")
        bc = _boundary(btab, shape, p_ref) if isinstance(btab, dict) else None
        obj, t = _geometry(g, D, bc)
        objects.append(obj)
        transforms[gname] = t

    zones = []
    for z in doc.get("refinement_zone", []):
        x0, x1 = get_entry(z, "start", "vec", size=3), get_entry(z, "end", "vec", size=3)
        level = get_entry(z, "max_refinement_level", "uint")
        like = z.get("transform_like")
        t = transforms.get(like) if like is not None else None
        if t is not None and not t.identity():
            # RefineZone::contains tests R^T S^-1 (x - t) against the box (config/config.hpp:82-85);
            # without rotation that is the world box t + S x0 .. t + S x1
            if t.rotation.any() or (t.scaling <= 0).any():
                raise NotImplementedError("refinement zones with a rotated or mirrored transform are not supported")
            x0, x1 = t.translation + t.scaling * x0, t.translation + t.scaling * x1
        zones.append(RefineZone(list(x0), list(x1), level))
    prm.zones = zones

    ic_data = None
    if x2p is None:
        if jump is None:
            ic_data = ("uniform", np.asarray(p_ref, np.float64))
        else:
            ic_data = ("jump", jump[0], jump[1], get_entry(ic, "value_neg", "vec", size=shape.E),
                       get_entry(ic, "value_pos", "vec", size=shape.E))
    spec = SceneSpec(shape, tuple(active), min_level, max_level, x2p or ic_x2p, domain_bc,
                     max_level_geom=max_level_geom, refinement_radius=radius, jump=jump, objects=objects,
                     zones=zones, diffuse_ic=diffuse, rho_ref=rho_ref, keep_ic_gas_density=False, ic=ic_data)
    if model == "multi" and D > 1 and objects and rho_ref is None:
        raise ConfigError("multiphase objects need reference densities")
    if builder not in ("host", "device", "auto"):
        raise ValueError("builder must be 'host', 'device' or 'auto'")
    tree = None
    if builder in ("device", "auto"):
        from .scene_gpu import build_tree_device

        try:
            tree = build_tree_device(spec)
        except NotImplementedError:
            if builder == "device":
                raise
    if tree is None:
        tree = build_tree(spec)
    run = RunSettings(name, io_interval, end_time, signal_time, steady_tol)
    return TomlCase(Case(tree, prm), spec, run, model, p_ref, vel_ref, rho_ref, ignored, objects)


def driver_for(tc: TomlCase, solver, out_dir: str, observers=(), **kw):
    """A DefaultDriver with the case's [run] settings, writing to `out_dir` (the reference writes to
    <project>/out/<scene.name>, config.cpp:31-37)."""
    from .driver import DefaultDriver

    r = tc.run
    return DefaultDriver(solver, r.name, os.path.join(out_dir, r.name), end_time=r.end_time,
                         io_interval=r.io_interval, observers=observers,
                         convergence_tol=max(r.convergence_tol, 0.0), signal_time=r.signal_time, **kw)
