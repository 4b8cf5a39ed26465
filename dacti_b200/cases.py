"""The benchmark and parity configurations as programmatic cases.

DACTI's TOML initial conditions only express uniform and single-jump states
(config/config.cpp:194-243), so the quadrant, shock-drop and random-batch cases are written here
as ``x2p`` functions over cell centres, the way ``Config::ic.x2p`` is consumed by
``Scene::init_domain`` (scene/scene.cpp:413-414). Coordinates are those of the reference: the root
box is centred at the origin with side ``max(active_size)``.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .casefile import Case, SolverParams
from .models import BcType, ModelId, ModelShape
from .scene import BoundarySpec, EllipseObject, SceneSpec, SphereObject, build_tree

ZG = BoundarySpec(BcType.ZERO_GRADIENT)


def _zg_box(D: int):
    return [(ZG, ZG) for _ in range(D)]


def lax_liu3(base_level: int = 6, levels: int = 3, thresholds=(0.02, 0.05), max_cfl: float = 0.5,
             model: ModelId = ModelId.EULER, mu: float = 0.0, prandtl: Optional[float] = None,
             domain_bc=None, limiter: int = 0) -> Case:
    """Config 1: 2D Euler Lax-Liu configuration 3 on the unit square, quadrants split at x=y=0.

    States (rho, u, v, p): TR (1.5,0,0,1.5), TL (0.5323,1.206,0,0.3), BL (0.138,1.206,1.206,0.029),
    BR (0.5323,0,1.206,0.3); outflow (zero-gradient) boundaries; density-weighted Laplacian
    indicator. The pair of thresholds (0.02, 0.05) is one for which the reference completes the run
    to t = 0.3 (tighter pairs make the reference itself produce NaN near t = 0.29).

    With ``model=ModelId.NAVIER_STOKES`` the same problem runs with constant viscosity ``mu`` and
    conductivity ``mu * cp / prandtl`` (model/navier_stokes.hpp:454-459). ``domain_bc`` replaces the
    zero-gradient faces with (neg, pos) BoundarySpec pairs per dimension; ``limiter`` selects the
    slope limiter by id.
    """
    shape = ModelShape(model, 2)

    def x2p(c: np.ndarray) -> np.ndarray:
        x, y = c[:, 0], c[:, 1]
        out = np.empty((c.shape[0], 4))
        tr = (x > 0) & (y > 0)
        tl = (x <= 0) & (y > 0)
        bl = (x <= 0) & (y <= 0)
        br = (x > 0) & (y <= 0)
        out[tr] = (1.5, 0.0, 0.0, 1.5)
        out[tl] = (0.5323, 1.206, 0.0, 0.3)
        out[bl] = (0.138, 1.206, 1.206, 0.029)
        out[br] = (0.5323, 0.0, 1.206, 0.3)
        return out

    spec = SceneSpec(shape, (1.0, 1.0), base_level, base_level + levels, x2p, domain_bc or _zg_box(2))
    prm = SolverParams(
        side_length=1.0, active_size=(1.0, 1.0), periodic=(False, False), max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=base_level + levels, min_level=base_level,
        weights=(1.0, 0.0, 0.0, 0.0),
        ns_mu=mu, ns_lambda=(mu * 1005.0 / prandtl) if prandtl else 0.0, limiter=limiter,
    )
    return Case(build_tree(spec), prm)


def riemann_batch(n_trees: int = 256, seed: int = 3, base_levels=(5, 8), extra_levels=(2, 4),
                  thresholds=(0.02, 0.05), max_cfl: float = 0.5) -> list:
    """Config 3: independent 2D Euler quadtree Riemann problems on the unit square, split at x = y = 0.

    Per tree, seeded: base grid 2^k x 2^k with k ~ U{base_levels}, 2-4 extra levels, and four quadrant
    states with rho ~ U(0.1, 2), p ~ U(0.02, 2), u, v ~ U(-1.5, 1.5); zero-gradient boundaries, CFL
    `max_cfl`, density-weighted Laplacian indicator. Each tree is one Integrator of the reference.
    """
    rng = np.random.default_rng(seed)
    out = []
    shape = ModelShape(ModelId.EULER, 2)
    for _ in range(n_trees):
        base = int(rng.integers(base_levels[0], base_levels[1] + 1))
        levels = int(rng.integers(extra_levels[0], extra_levels[1] + 1))
        q = np.empty((4, 4))
        q[:, 0] = rng.uniform(0.1, 2.0, 4)
        q[:, 1] = rng.uniform(-1.5, 1.5, 4)
        q[:, 2] = rng.uniform(-1.5, 1.5, 4)
        q[:, 3] = rng.uniform(0.02, 2.0, 4)

        def x2p(c: np.ndarray, q=q) -> np.ndarray:
            x, y = c[:, 0], c[:, 1]
            k = np.where(x > 0, np.where(y > 0, 0, 3), np.where(y > 0, 1, 2))
            return q[k].copy()

        spec = SceneSpec(shape, (1.0, 1.0), base, base + levels, x2p, _zg_box(2))
        prm = SolverParams(
            side_length=1.0, active_size=(1.0, 1.0), periodic=(False, False), max_cfl=max_cfl, max_dt=1.0,
            error_threshold=thresholds, max_level=base + levels, min_level=base, weights=(1.0, 0.0, 0.0, 0.0),
        )
        out.append(Case(build_tree(spec), prm))
    return out


def normal_shock(rho1: float, p1: float, mach: float, gamma: float = 1.4, P0: float = 0.0):
    """Post-shock (rho, u, p) behind a normal shock moving into gas at rest.

    Same relations as config::compute_normal_shock (config/util.hpp:135-150).
    """
    c1 = math.sqrt(gamma * (p1 + P0) / rho1)
    r_ratio = 1.0 - 2.0 / (gamma + 1) * (1 - 1 / (mach * mach))
    r2 = rho1 / r_ratio
    u2 = 2.0 / (gamma + 1) * (mach - 1 / mach) * c1
    p2 = p1 * (((2 * P0 / p1 + 1) * (1 - r_ratio) * gamma + 1 + r_ratio) / ((r_ratio - 1) * gamma + 1 + r_ratio))
    return r2, u2, p2


def shock_drop_spec(*args, **kw):
    """(SceneSpec, SolverParams) of shock_drop, for builders other than the host one."""
    return shock_drop(*args, _spec_only=True, **kw)


def shock_drop(dims: int = 3, base_level: int = 6, levels: int = 4, length: float = 8e-3, aspect: int = 2,
               drop_radius: float = 0.5e-3, shock_x: float = -1.0e-3, mach: float = 1.5,
               thresholds=(0.02, 0.05), max_cfl: float = 0.25, weights: Optional[tuple] = None,
               mu: tuple = (0.0, 0.0), conductivity: tuple = (0.0, 0.0), sigma: float = 0.0,
               _spec_only: bool = False) -> Case:
    """Config 2: five-equation air-water shock-drop.

    Domain ``length`` x ``length/aspect`` (x ``length/aspect``) with a ``2^base_level`` cell root
    grid along x, ``levels`` refinement levels; water drop (stiffened gas gamma=4.4, pi_inf=6e8 Pa,
    rho=1000) of ``drop_radius`` at the origin in air (gamma=1.4, rho=1.2, p=1e5); a Mach ``mach``
    planar shock at x = ``shock_x`` moving in +x with the Rankine-Hugoniot post-shock state behind
    it; volume fraction smeared with a tanh over the finest cell size. The inflow face carries the
    post-shock state; all other faces are zero-gradient. Surface tension and viscosity are zero.
    The CFL target 0.25 is the one of the reference's own cases/shockDrop3d.toml; at 0.5 the 3D
    reference run floors the water pressure once the shock reaches the drop. ``mu``,
    ``conductivity`` (water, air) and ``sigma`` switch on the viscous, heat and surface-tension terms
    of model/multi.hpp.
    """
    shape = ModelShape(ModelId.MULTI, dims)
    E = shape.E
    rho_w, rho_a, p0 = 1000.0, 1.2, 1.0e5
    r2, u2, p2 = normal_shock(rho_a, p0, mach)
    active = [length] + [length / aspect] * (dims - 1)

    def state(rho_air: float, u: float, p: float) -> np.ndarray:
        s = np.zeros(E)
        s[0] = 0.0          # alpha1 rho1 (water)
        s[1] = rho_air      # alpha2 rho2 (air)
        s[2] = u
        s[shape.ip] = p
        s[shape.ia] = 0.0
        return s

    post = state(r2, u2, p2)
    pre = state(rho_a, 0.0, p0)

    def x2p(c: np.ndarray) -> np.ndarray:
        out = np.where((c[:, 0] > shock_x)[:, None], pre[None, :], post[None, :])
        return out.copy()

    inflow = BoundarySpec(BcType.INFLOW, list(post), None, 0.0)
    dbc = [(inflow, ZG)] + [(ZG, ZG) for _ in range(dims - 1)]
    spec = SceneSpec(
        shape, active, base_level, base_level + levels, x2p, dbc,
        jump=(0, shock_x),
        objects=[SphereObject((0.0, 0.0, 0.0), drop_radius, "droplet")],
        diffuse_ic=True, rho_ref=(rho_w, rho_a), ic=("jump", 0, shock_x, post, pre),
    )
    if weights is None:
        weights = (1e-3, 1.0) + (0.0,) * dims + (3e-6, 1.0)
    prm = SolverParams(
        side_length=length, active_size=active, periodic=[False] * dims, max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=base_level + levels, min_level=base_level, weights=weights,
        gamma1=4.4, gamma2=1.4, P1=6.0e8, P2=0.0, mu1=mu[0], mu2=mu[1], lambda1=conductivity[0],
        lambda2=conductivity[1], sigma=sigma,
    )
    if _spec_only:
        return spec, prm
    return Case(build_tree(spec), prm)


def box_blast(base_level: int = 3, levels: int = 2, thresholds=(0.02, 0.05), max_cfl: float = 0.5,
              p_in: float = 5.0, model: ModelId = ModelId.EULER, mu: float = 0.0, prandtl: float = 0.72,
              domain_bc=None) -> Case:
    """2D Euler / Navier-Stokes blast in the unit box: rho 1.5, p = ``p_in`` inside a disc of radius
    0.2 at (0.1, -0.05), rho 1, p 1 outside, uniform drift (0.2, -0.1). Its waves reach every face of
    the box within one time unit, which exercises the wall treatments (integrator/boundary.hpp:
    76-89, 128-142): ``domain_bc`` gives (neg, pos) BoundarySpec pairs per dimension, freeslip
    on x and noslip on y by default. (The Lax-Liu configuration 3 runs into the reference's wall
    boundary fluxes at Mach ~1 and breaks down with NaN after a few steps, so it is not used here.)"""
    shape = ModelShape(model, 2)

    def x2p(c: np.ndarray) -> np.ndarray:
        inside = np.hypot(c[:, 0] - 0.1, c[:, 1] + 0.05) < 0.2
        out = np.empty((c.shape[0], 4))
        out[:, 0] = np.where(inside, 1.5, 1.0)
        out[:, 1] = 0.2
        out[:, 2] = -0.1
        out[:, 3] = np.where(inside, p_in, 1.0)
        return out

    if domain_bc is None:
        domain_bc = [(BoundarySpec(BcType.FREESLIP),) * 2, (BoundarySpec(BcType.NOSLIP),) * 2]
    spec = SceneSpec(shape, (1.0, 1.0), base_level, base_level + levels, x2p, domain_bc)
    prm = SolverParams(
        side_length=1.0, active_size=(1.0, 1.0), periodic=(False, False), max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=base_level + levels, min_level=base_level,
        weights=(1.0, 0.0, 0.0, 0.0), ns_mu=mu, ns_lambda=mu * 1005.0 / prandtl if mu else 0.0,
    )
    return Case(build_tree(spec), prm)


def periodic_blob(base_level: int = 4, levels: int = 2, thresholds=(0.02, 0.05), max_cfl: float = 0.5,
                  refine: bool = True) -> Case:
    """2D Euler on a doubly periodic unit square: a dense square (rho 2 inside |x|,|y| < 0.15, else 1)
    advected with (u, v) = (1, 0.5) at p = 1. Exercises the periodic neighbour wrap of
    Domain::find (integrator/domain.hpp:65-82), the shifted neighbour centre of the flux stage
    (impl/flux.hpp:67-78) and of the estimator (impl/adaptive_refinement.hpp:51-57).
    With refine=False the tree stays at the base level (min = max level)."""
    shape = ModelShape(ModelId.EULER, 2)

    def x2p(c: np.ndarray) -> np.ndarray:
        inside = (np.abs(c[:, 0]) < 0.15) & (np.abs(c[:, 1]) < 0.15)
        out = np.empty((c.shape[0], 4))
        out[:, 0] = np.where(inside, 2.0, 1.0)
        out[:, 1] = 1.0
        out[:, 2] = 0.5
        out[:, 3] = 1.0
        return out

    max_level = base_level + (levels if refine else 0)
    spec = SceneSpec(shape, (1.0, 1.0), base_level, max_level, x2p, [None, None])
    prm = SolverParams(
        side_length=1.0, active_size=(1.0, 1.0), periodic=(True, True), max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=max_level, min_level=base_level, weights=(1.0, 0.0, 0.0, 0.0),
    )
    return Case(build_tree(spec), prm)


def smooth_periodic(base_level: int = 3, levels: int = 2, thresholds=(0.02, 0.05), max_cfl: float = 0.5,
                    limiter: int = 0) -> Case:
    """2D Euler on a doubly periodic unit square with every primitive varying smoothly: a periodic
    Gaussian density bump of width 0.1 on a background of sines, sheared velocity, pressure wave.
    No two neighbouring cells hold equal values, so the slope limiters whose formula is 0/0 on
    equal slopes (van Leer, van Albada 2 in integrator/slope_limiters.hpp) stay finite; the
    reference produces NaN on them wherever the flow is piecewise constant."""
    shape = ModelShape(ModelId.EULER, 2)
    tp = 2.0 * math.pi

    def x2p(c: np.ndarray) -> np.ndarray:
        x, y = c[:, 0], c[:, 1]
        bump = np.exp(-(np.sin(math.pi * x) ** 2 + np.sin(math.pi * y) ** 2) / 0.01)
        out = np.empty((c.shape[0], 4))
        out[:, 0] = 1.0 + 0.5 * bump + 0.1 * np.sin(tp * x + 0.3) * np.sin(tp * y + 1.1) + 0.05 * np.cos(tp * (x + 2 * y))
        out[:, 1] = 0.3 + 0.1 * np.cos(tp * y + 0.4) + 0.02 * np.sin(tp * (x - y) + 0.9)
        out[:, 2] = -0.2 + 0.1 * np.sin(tp * x + 0.2) + 0.03 * np.cos(tp * (2 * x + y) + 0.5) + 0.02 * np.sin(tp * y + 0.7)
        out[:, 3] = 1.0 + 0.1 * np.sin(tp * (x - y) + 0.6) + 0.03 * np.cos(tp * (x + y) + 0.8) + 0.2 * bump
        return out

    spec = SceneSpec(shape, (1.0, 1.0), base_level, base_level + levels, x2p, [None, None])
    prm = SolverParams(
        side_length=1.0, active_size=(1.0, 1.0), periodic=(True, True), max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=base_level + levels, min_level=base_level,
        weights=(1.0, 0.0, 0.0, 0.0), limiter=limiter,
    )
    return Case(build_tree(spec), prm)


def osc_drop(base_level: int = 4, levels: int = 2, thresholds=(1e-3, 1e-2), max_cfl: float = 0.4,
             conductivity: tuple = (0.0, 0.0), velocity: float = 0.0, sigma: float = 0.1, oh: float = 0.01,
             rho_gas: float = 1e-3) -> Case:
    """2D oscillating drop in the non-dimensional units of the reference's cases/oscDrop.toml:
    2 x 2 box, elliptic drop (a = 0.2, b = 0.12) of fluid 1 (rho 1, gamma 6.12, P0 500) in fluid 2
    (rho 1e-3, gamma 1.4), p = 1 at rest, sigma = 0.1, Oh = 0.01 with L = 0.15825 and viscosity ratio
    10 (mu1 = sqrt(rho1 sigma L) Oh, model/multi.hpp:531-535), tanh-smeared interface,
    zero-gradient boundaries. Exercises surface tension (curvature, smoothing, source) and the
    viscous terms of the five-equation model. ``velocity`` translates everything along x;
    ``rho_gas`` replaces the gas density."""
    shape = ModelShape(ModelId.MULTI, 2)
    rho1, rho2, L = 1.0, rho_gas, 0.15825
    mu1 = math.sqrt(rho1 * sigma * L) * oh

    def x2p(c: np.ndarray) -> np.ndarray:
        out = np.zeros((c.shape[0], 6))
        out[:, 1] = rho2
        out[:, 2] = velocity
        out[:, 4] = 1.0
        return out

    spec = SceneSpec(shape, (2.0, 2.0), base_level, base_level + levels, x2p, _zg_box(2),
                     objects=[EllipseObject((0.0, 0.0), (0.2, 0.12), "droplet")], diffuse_ic=True,
                     rho_ref=(rho1, rho2))
    prm = SolverParams(
        side_length=2.0, active_size=(2.0, 2.0), periodic=(False, False), max_cfl=max_cfl, max_dt=5e-3,
        error_threshold=thresholds, max_level=base_level + levels, min_level=base_level,
        weights=(1.0, 0.0, 0.0, 0.0, 0.0, 1.0), gamma1=6.12, gamma2=1.4, P1=500.0, P2=0.0,
        mu1=mu1, mu2=mu1 / 10.0, lambda1=conductivity[0], lambda2=conductivity[1], sigma=sigma,
    )
    return Case(build_tree(spec), prm)


def cylinder_ns_spec(*args, **kw):
    """(SceneSpec, SolverParams) of cylinder_ns, for builders other than the host one."""
    return cylinder_ns(*args, _spec_only=True, **kw)


def cylinder_ns(mach: float = 0.3, base_level: int = 5, levels: int = 3, reynolds: float = 200.0,
                prandtl: float = 0.72, thresholds=(5e-3, 1e-2), max_cfl: float = 0.4,
                weights=(1.0, 0.01, 0.01, 1e-5), diameter: float = 1.0, center=(-10.0, 0.0),
                _spec_only: bool = False) -> Case:
    """2D Navier-Stokes flow past a cylinder: domain 40 x 20 (root side 40, so a 2^base_level x
    2^(base_level-1) base grid), a solid circle of the given diameter with a no-slip wall, inflow of air
    (rho 1.2, p 101325) at the given Mach number on x-, outflow on x+, free-slip walls on y. The
    viscosity follows the reference's Navier-Stokes dict (model/navier_stokes.hpp:120-134) with the
    diameter as length: mu = rho |u| D / Re, lambda = mu cp / Pr. Cells next to the cylinder sit at the
    finest level."""
    shape = ModelShape(ModelId.NAVIER_STOKES, 2)
    rho, p = 1.2, 101325.0
    u = mach * math.sqrt(1.4 * p / rho)
    mu = rho * u * diameter / reynolds
    ref = [rho, u, 0.0, p]

    def x2p(c: np.ndarray) -> np.ndarray:
        return np.tile(ref, (c.shape[0], 1))

    out = [0.0, 0.0, 0.0, p]
    domain_bc = [(BoundarySpec(BcType.INFLOW, ref), BoundarySpec(BcType.OUTFLOW, out)),
                 (BoundarySpec(BcType.FREESLIP), BoundarySpec(BcType.FREESLIP))]
    wall = SphereObject(center, 0.5 * diameter, "solid", BoundarySpec(BcType.NOSLIP))
    top = base_level + levels
    spec = SceneSpec(shape, (40.0, 20.0), base_level, top, x2p, domain_bc, max_level_geom=top, objects=[wall],
                     ic=("uniform", np.asarray(ref, np.float64)))
    prm = SolverParams(
        side_length=40.0, active_size=(40.0, 20.0), periodic=(False, False), max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=top, min_level=base_level, weights=weights,
        ns_mu=mu, ns_lambda=mu * 1005.0 / prandtl,
    )
    if _spec_only:
        return spec, prm
    return Case(build_tree(spec), prm)


def blast3d(base_level: int = 3, levels: int = 2, thresholds=(0.02, 0.05), max_cfl: float = 0.5,
            model: ModelId = ModelId.EULER, mu: float = 0.0, prandtl: float = 0.72) -> Case:
    """3D Euler / Navier-Stokes blast in the unit cube: rho 1.5, p 3 inside a sphere of radius 0.25 at
    (0.1, -0.05, 0.05), rho 1, p 1 outside, uniform drift (0.2, -0.1, 0.05). Free-slip walls on x,
    no-slip walls on y, periodic in z: the 3D neighbour search, hanging faces in three directions, both
    wall treatments and the periodic wrap in one case."""
    shape = ModelShape(model, 3)

    def x2p(c: np.ndarray) -> np.ndarray:
        inside = np.sqrt((c[:, 0] - 0.1) ** 2 + (c[:, 1] + 0.05) ** 2 + (c[:, 2] - 0.05) ** 2) < 0.25
        out = np.empty((c.shape[0], 5))
        out[:, 0] = np.where(inside, 1.5, 1.0)
        out[:, 1] = 0.2
        out[:, 2] = -0.1
        out[:, 3] = 0.05
        out[:, 4] = np.where(inside, 3.0, 1.0)
        return out

    domain_bc = [(BoundarySpec(BcType.FREESLIP),) * 2, (BoundarySpec(BcType.NOSLIP),) * 2, None]
    spec = SceneSpec(shape, (1.0, 1.0, 1.0), base_level, base_level + levels, x2p, domain_bc)
    prm = SolverParams(
        side_length=1.0, active_size=(1.0, 1.0, 1.0), periodic=(False, False, True), max_cfl=max_cfl, max_dt=1.0,
        error_threshold=thresholds, max_level=base_level + levels, min_level=base_level,
        weights=(1.0, 0.0, 0.0, 0.0, 0.0), ns_mu=mu, ns_lambda=mu * 1005.0 / prandtl if mu else 0.0,
    )
    return Case(build_tree(spec), prm)
