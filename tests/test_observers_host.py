"""AeroForce (driver/observer/aero_force.hpp) and the point location it uses, on synthetic leaves:
a linear pressure field gives the buoyancy-like force grad(p) times the sampled area."""
import math

import numpy as np

from dacti_b200.casefile import Snapshot
from dacti_b200.driver import AeroForce, find_in_tree, locate
from dacti_b200.htg import NodeTable
from dacti_b200.models import BcType, ModelId, ModelShape
from dacti_b200.scene import BoundarySpec, EllipseObject, PolygonObject, SphereObject


class _S:
    side_length = 2.0
    shape = ModelShape(ModelId.EULER, 2)


def _uniform(level, side, p_of_x):
    n = 1 << level
    h = side / n
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    c = np.stack([(ii.ravel() + 0.5) * h - side / 2, (jj.ravel() + 0.5) * h - side / 2], axis=1)
    m = c.shape[0]
    p = np.tile([1.2, 0.0, 0.0, 0.0], (m, 1))
    p[:, 3] = p_of_x(c)
    z = np.zeros(m)
    return Snapshot(2, 4, 0, 0, 0, m, 0.0, 0.0, 0.0, np.full(m, level, np.int32), np.zeros(m, np.int32), c, z, p, p,
                    z, z, z)


def test_locate_finds_the_containing_leaf():
    snap = _uniform(4, 2.0, lambda c: np.zeros(c.shape[0]))
    rng = np.random.default_rng(0)
    pts = rng.uniform(-0.999, 0.999, (200, 2))
    idx = locate(snap, 2.0, pts)
    h = 2.0 / 16
    assert (idx >= 0).all() and (np.abs(snap.center[idx] - pts) <= h / 2 + 1e-12).all()
    assert locate(snap, 2.0, np.array([[1.5, 0.0]]))[0] == -1


def test_aero_force_of_a_linear_pressure_field():
    G, p0, rho, u = 3.0, 100.0, 1.2, 2.0
    wall = BoundarySpec(BcType.NOSLIP)
    snap = _uniform(9, 2.0, lambda c: p0 - G * c[:, 0] + 0.5 * G * c[:, 1])
    q = 0.5 * rho * u * u
    for obj, area in [(SphereObject((0.1, -0.05), 0.3, "solid", wall), None),
                      (EllipseObject((0.0, 0.1), (0.4, 0.2), "solid", wall, 25.0), None),
                      (PolygonObject([[0, 0.3], [0.3, 0], [0, -0.3], [-0.3, 0]], "solid", wall), None)]:
        ob = AeroForce([obj], [rho, u, 0.0, p0], [u, 0.0], n_segments=512, convention="fluid")
        cl, cd = ob.observe(_S, snap)
        # exact sums of the pressure at the sample points (cell values differ by at most G h / 2)
        dp = -G * ob.pts[:, 0] + 0.5 * G * ob.pts[:, 1]
        fx = -(dp / q * ob.area * ob.nrm[:, 0]).sum()
        fy = -(dp / q * ob.area * ob.nrm[:, 1]).sum()
        assert math.isclose(cd, fx, rel_tol=1e-2) and math.isclose(cl, fy, rel_tol=1e-2), (cd, fx, cl, fy)
        # ... which is grad(p) times the enclosed area, to first order in the 0.01 offset
        ring = ob.pts - 0.01 * ob.nrm
        a = 0.5 * abs((ring[:, 0] * np.roll(ring[:, 1], -1) - np.roll(ring[:, 0], -1) * ring[:, 1]).sum())
        assert math.isclose(cd, G * a / q, rel_tol=0.1) and math.isclose(cl, -0.5 * G * a / q, rel_tol=0.1)
        cp, surf = ob.fields(_S, snap)
        assert surf.sum() > 0 and (cp[surf == 0] == 0).all()


def _full_tree(level, side, p_of_x):
    """A complete quadtree to `level` as a node table (slot 0 null, slot 1 root), leaves' p from p_of_x."""
    parent, children, lv, flags, centers = [0, 0], [[0] * 4, [0] * 4], [0, 0], [0, 3], [[0.0, 0.0], [0.0, 0.0]]
    frontier = [1]
    for l in range(level):
        nxt = []
        h = side / (1 << (l + 1))
        for x in frontier:
            flags[x] = 2  # active, no longer a leaf
            for k in range(4):
                c = [centers[x][0] + (0.5 if k & 1 else -0.5) * h, centers[x][1] + (0.5 if k & 2 else -0.5) * h]
                children[x][k] = len(parent)
                parent.append(x)
                children.append([0] * 4)
                lv.append(l + 1)
                flags.append(3)
                centers.append(c)
                nxt.append(len(parent) - 1)
        frontier = nxt
    n = len(parent)
    p = np.zeros((n, 4))
    ctr = np.array(centers)
    p[:, 0] = 1.2
    p[:, 3] = p_of_x(ctr)
    return NodeTable(2, np.array(parent, np.int32), np.array(children, np.int32), np.array(lv, np.int32),
                     np.array(flags, np.uint32), p, np.zeros((n, 4))), ctr


def test_find_in_tree_is_domain_find():
    nodes, ctr = _full_tree(4, 2.0, lambda c: np.zeros(c.shape[0]))
    rng = np.random.default_rng(1)
    pts = rng.uniform(-0.999, 0.999, (100, 2))
    idx = find_in_tree(nodes, 2.0, (2.0, 2.0), (False, False), pts)
    h = 2.0 / 16
    assert (nodes.flags[idx] & 1).all() and (np.abs(ctr[idx] - pts) <= h / 2 + 1e-12).all()
    assert find_in_tree(nodes, 2.0, (2.0, 2.0), (False, False), np.array([[1.5, 0.0]]))[0] == 0
    assert find_in_tree(nodes, 2.0, (2.0, 2.0), (True, False), np.array([[1.5, 0.0]]))[0] != 0


def test_aero_force_reference_convention_samples_inside_the_body():
    """aero_force.hpp:47-50 and 92-100: samples 0.01 against rotaten90 of the tangent (into the body of a
    counter-clockwise outline), Cl/Cd = sum Cp area n_s; on a linear pressure field that is minus the
    fluid-side force to first order in the offsets."""
    G, p0, rho, u = 3.0, 100.0, 1.2, 2.0
    wall = BoundarySpec(BcType.NOSLIP)
    f = lambda c: p0 - G * c[:, 0] + 0.5 * G * c[:, 1]
    nodes, _ = _full_tree(7, 2.0, f)
    snap = _uniform(7, 2.0, f)

    class S(_S):
        class params:
            active_size, periodic = (2.0, 2.0), (False, False)

        @staticmethod
        def tree_nodes():
            return nodes

    obj = SphereObject((0.1, -0.05), 0.3, "solid", wall)
    ref = AeroForce([obj], [rho, u, 0.0, p0], [u, 0.0], n_segments=256)
    flu = AeroForce([obj], [rho, u, 0.0, p0], [u, 0.0], n_segments=256, convention="fluid")
    # samples sit inside the circle for the reference convention, outside for the fluid one
    r_ref = np.hypot(ref.pts[:, 0] - 0.1, ref.pts[:, 1] + 0.05)
    r_flu = np.hypot(flu.pts[:, 0] - 0.1, flu.pts[:, 1] + 0.05)
    assert (r_ref < 0.3).all() and (r_flu > 0.3).all()
    cl, cd = ref.observe(S, snap)
    cl_f, cd_f = flu.observe(S, snap)
    assert math.isclose(cd, -cd_f, rel_tol=0.1) and math.isclose(cl, -cl_f, rel_tol=0.1), (cd, cd_f, cl, cl_f)
