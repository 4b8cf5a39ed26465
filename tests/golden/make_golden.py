"""Generates the golden fixtures of the parity tests by running the reference solver.

Each fixture is a case file (the exact initial tree handed to both solvers) and the reference's
snapshots of every active cell at the listed global steps, produced by DACTI's own Integrator
compiled from its sources (oracle/_ref/dacti_ref_runner, single thread, no FMA contraction).

    python tests/golden/make_golden.py        # rewrites tests/golden/*.case and *.snap
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dacti_b200 import cases  # noqa: E402
from dacti_b200.casefile import write_case  # noqa: E402
from dacti_b200.models import BcType, ModelId  # noqa: E402
from dacti_b200.scene import BoundarySpec  # noqa: E402

# Fixed-state conditions sit on the negative faces: the reference's boundary flux passes the
# boundary state as the left Riemann state on every face (integrator/boundary.hpp:143-149), which
# is unstable on positive faces for these inflow states.
OUT = BoundarySpec(BcType.OUTFLOW, (0.0, 0.0, 0.0, 1.0))
OPEN_A = [(BoundarySpec(BcType.INFLOW, (1.0, 0.4, -0.1, 1.0), None, 0.3), OUT),
          (BoundarySpec(BcType.INFLOW_R, (1.2, 0.0, 0.3, 1.1), None, 0.0), OUT)]
OPEN_B = [(BoundarySpec(BcType.DIRICHLET, (1.0, 0.2, -0.1, 1.0)), BoundarySpec(BcType.ZERO_GRADIENT)),
          (BoundarySpec(BcType.INFLOW, (1.1, 0.0, 0.2, 1.2), None, 0.0), OUT)]

RUNNER = os.path.join(ROOT, "oracle", "_ref", "dacti_ref_runner")

# name -> (case factory, global steps, check steps)
GOLDEN = {
    "euler2": (lambda: cases.lax_liu3(base_level=3, levels=2), 6, [2, 6]),
    "ns2": (lambda: cases.lax_liu3(base_level=3, levels=2, model=ModelId.NAVIER_STOKES, mu=2e-3, prandtl=0.72), 6,
            [6]),
    "multi2": (lambda: cases.shock_drop(dims=2, base_level=4, levels=2), 4, [0, 4]),
    "multi3": (lambda: cases.shock_drop(dims=3, base_level=3, levels=1), 2, [0, 2]),
    "euler2_periodic": (lambda: cases.periodic_blob(base_level=3, levels=2), 6, [6]),
    # 3D Euler and Navier-Stokes (walls, periodic z, hanging faces in three directions)
    "euler3": (lambda: cases.blast3d(base_level=3, levels=1), 4, [2, 4]),
    "ns3": (lambda: cases.blast3d(base_level=3, levels=1, model=ModelId.NAVIER_STOKES, mu=2e-3), 4, [4]),
    # boundary conditions: freeslip / noslip walls, inflow with fade-in, inflow_r, Dirichlet, outflow
    "euler2_walls": (lambda: cases.box_blast(base_level=3, levels=2), 10, [5, 10]),
    "euler2_open_a": (lambda: cases.box_blast(base_level=3, levels=2, domain_bc=OPEN_A), 10, [5, 10]),
    "euler2_open_b": (lambda: cases.box_blast(base_level=3, levels=2, domain_bc=OPEN_B), 10, [10]),
    "ns2_walls": (lambda: cases.box_blast(base_level=3, levels=2, model=ModelId.NAVIER_STOKES, mu=2e-3), 10, [10]),
    # slope limiters other than minmod (integrator/slope_limiters.hpp:18-57)
    **{f"euler2_lim{k}": (lambda k=k: cases.smooth_periodic(base_level=4, levels=2, limiter=k), 6, [6])
       for k in range(1, 7)},
    # viscosity and heat conduction of the five-equation model
    "multi2_visc": (lambda: cases.shock_drop(dims=2, base_level=4, levels=2, mu=(1e-3, 1.8e-5),
                                             conductivity=(0.6, 0.026)), 4, [4]),
    # surface tension: a translating drop in the units of the reference's oscillating-drop case. With
    # the gas density of 1e-3 the reference reaches NaN in its second global step (its fixed floor
    # alpha1 rho1 >= 1e-3 doubles the gas density), so that fixture holds the constructed state:
    # smoothed volume fraction, normals and curvature, bit for bit.
    "multi2_tension": (lambda: cases.osc_drop(velocity=0.5), 0, [0]),
    # ... and with a gas of density 0.5 it runs for four steps before the curvature, converted to an
    # unsigned integer in the surface-tension Jacobian (model/multi.hpp:126), blows up; two are checked.
    "multi2_tension_run": (lambda: cases.osc_drop(velocity=0.5, rho_gas=0.5), 2, [1, 2]),
}


def generate(name: str) -> None:
    factory, steps, checks = GOLDEN[name]
    case = factory()
    path = os.path.join(HERE, f"{name}.case")
    write_case(case, path)
    subprocess.run([RUNNER, path, os.path.join(HERE, name), str(steps), "--check", ",".join(map(str, checks))],
                   check=True, capture_output=True, env=dict(os.environ, OMP_NUM_THREADS="1"))


if __name__ == "__main__":
    for n in (sys.argv[1:] or GOLDEN):
        generate(n)
        print(n)
