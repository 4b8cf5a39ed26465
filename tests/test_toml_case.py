"""TOML case files (config/config.cpp:10-243 restated in dacti_b200/toml_case.py): defaults, the
models' dict() constants, initial conditions, boundary conditions, geometry, refinement zones, the
get_entry type rules, and the reference parser's quirks."""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN
from dacti_b200.casefile import read_case, write_case
from dacti_b200.models import BcType, F_ACTIVE, F_LEAF
from dacti_b200.toml_case import ConfigError, load_toml_case

TOML = os.path.join(GOLDEN, "toml")


def _path(name):
    return os.path.join(TOML, f"{name}.toml")


def _write(tmp_path, text, name="c"):
    p = tmp_path / f"{name}.toml"
    p.write_text(text)
    return str(p)


BASE = """
[scene]
name = "t"
domain_size = [1.0, 1.0]
[run]
print_interval = 0.1
end_time = 0.2
[integrator]
min_refinement_level = 3
max_refinement_level = 4
error_threshold = [0.02, 0.05]
max_cfl = 0.5
[model.reference_values]
rho = 1.0
vel = [0.5, 0.0]
p = 1.0
[initial_condition]
type = "uniform"
[boundary_conditions.X]
type = "periodic"
[boundary_conditions.Y]
type = "periodic"
"""


def _write_text(text):
    import tempfile

    f = tempfile.NamedTemporaryFile("w", suffix=".toml", delete=False)
    f.write(text)
    f.close()
    return f.name


def _leaves(tc):
    t = tc.case.tree
    return t.leaf_mask()


def test_defaults_and_euler_reference_state(tmp_path):
    tc = load_toml_case(_write(tmp_path, BASE))
    prm = tc.case.params
    assert tc.model == "euler" and tc.case.shape.dims == 2
    assert prm.max_dt == 0.1  # integrator.max_dt defaults to run.print_interval
    assert tuple(prm.weights) == (1.0, 1.0, 1.0, 1.0)  # error_weights default ones
    assert tc.run.signal_time == -1.0 and tc.run.convergence_tol == -1.0
    assert list(prm.periodic) == [True, True] and tc.case.tree.bcs == []
    assert np.array_equal(tc.p_ref, [1.0, 0.5, 0.0, 1.0])
    t = tc.case.tree
    lm = _leaves(tc)
    assert (t.level[lm] == 3).all() and lm.sum() == 64
    assert np.allclose(t.p[lm], [1.0, 0.5, 0.0, 1.0])


def test_type_rules(tmp_path):
    # scalars must be floats, integers integers, vectors float arrays of the right length
    with pytest.raises(ConfigError, match="floating point"):
        load_toml_case(_write(tmp_path, BASE.replace("p = 1.0", "p = 1")))
    with pytest.raises(ConfigError, match="int"):
        load_toml_case(_write(tmp_path, BASE.replace("min_refinement_level = 3", "min_refinement_level = 3.0")))
    with pytest.raises(ConfigError, match="Length"):
        load_toml_case(_write(tmp_path, BASE.replace("vel = [0.5, 0.0]", "vel = [0.5, 0.0, 0.0]")))
    with pytest.raises(ConfigError, match=r"vel\[1\]"):
        load_toml_case(_write(tmp_path, BASE.replace("vel = [0.5, 0.0]", "vel = [0.5, 0]")))
    with pytest.raises(ConfigError, match="Couldn't find entry for run.end_time"):
        load_toml_case(_write(tmp_path, BASE.replace("end_time = 0.2", "")))


def test_uniform_fixed_uses_reference_state(tmp_path):
    text = BASE.replace('type = "uniform"', 'type = "uniform"\nvalue = "fixed"')
    with pytest.raises(ConfigError, match="fixed_value"):
        load_toml_case(_write(tmp_path, text))
    tc = load_toml_case(_write(tmp_path, text.replace('value = "fixed"',
                                                      'value = "fixed"\nfixed_value = [2.0, 0.0, 0.0, 3.0]')))
    lm = _leaves(tc)
    assert np.allclose(tc.case.tree.p[lm], tc.p_ref)  # config.cpp:208-210 returns p_ref
    assert "initial_condition.fixed_value" in tc.ignored
    with pytest.raises(ConfigError, match="Unknown uniform value type"):
        load_toml_case(_write(tmp_path, BASE.replace('type = "uniform"', 'type = "uniform"\nvalue = "other"')))
    with pytest.raises(ConfigError, match="Unknown initial condition type"):
        load_toml_case(_write(tmp_path, BASE.replace('type = "uniform"', 'type = "ramp"')))


def test_boundary_conditions(tmp_path):
    text = BASE.replace('[boundary_conditions.X]\ntype = "periodic"', """
[boundary_conditions.X.neg]
type = "inflow"
fade_in = 0.25
[boundary_conditions.X.pos]
type = "outflow"
""").replace('[boundary_conditions.Y]\ntype = "periodic"', """
[boundary_conditions.Y.neg]
type = "noslip"
[boundary_conditions.Y.pos]
type = "inflow_r"
value = [2.0, 0.0, -0.5, 3.0]
""")
    tc = load_toml_case(_write(tmp_path, text))
    b = tc.case.tree.bcs
    assert [x.type for x in b] == [BcType.INFLOW, BcType.OUTFLOW, BcType.NOSLIP, BcType.INFLOW_R]
    assert np.allclose(b[0].p_in, tc.p_ref) and b[0].fade_in == 0.25
    assert np.allclose(b[1].p_in, [0.0, 0.0, 0.0, 1.0])  # outflow keeps p_ref[ip] only
    assert np.allclose(b[2].normal, [0.0, 1.0])  # -unit(dim) * (2 dir - 1)
    assert np.allclose(b[3].p_in, [2.0, 0.0, -0.5, 3.0])
    assert list(tc.case.params.periodic) == [False, False]
    # inflow_r faces refine to the maximum level (scene.cpp:177-189)
    t = tc.case.tree
    lm = _leaves(tc)
    top = lm & (t.center[:, 1] > 0.5 - 1.0 / 8)
    assert (t.level[top] == 4).all()
    with pytest.raises(ConfigError, match="illegal bc type"):
        load_toml_case(_write(tmp_path, text.replace('type = "noslip"', 'type = "wall"')))
    with pytest.raises(ConfigError, match="only 'periodic'"):
        load_toml_case(_write(tmp_path, BASE.replace('[boundary_conditions.Y]\ntype = "periodic"',
                                                     '[boundary_conditions.Y]\ntype = "noslip"')))


def test_multiphase_drop_constants_and_quirks():
    tc = load_toml_case(_path("drop2d"))
    prm = tc.case.params
    assert tc.model == "multi"
    assert prm.sigma == 0.05 and prm.gamma1 == 5.5 and prm.P1 == 400.0
    assert prm.gamma2 == 1.4 and prm.P2 == 0.0  # no fluid_2 table: defaults
    mu1 = math.sqrt(1.0 * 0.05 * 0.2) * 0.02  # Oh branch, model/multi.hpp:531-535
    assert prm.mu1 == mu1 and prm.mu2 == mu1 / 20.0
    assert prm.cv1 == 4181.0 / 6.12  # cv from the default gammas (model/multi.hpp:57-58)
    # diffuse_ic is read from the wrong path by the reference: sharp 0/1 volume fractions
    assert tc.ignored == ["initial_condition.diffuse_ic"]
    t = tc.case.tree
    lm = _leaves(tc)
    a = t.p[lm, 5]
    assert set(np.unique(a)) == {0.0, 1.0}
    # the rotated, translated ellipse: x = R S y + t
    c = t.center[lm]
    th = math.radians(30.0)
    y = c - [0.1, -0.05]
    yb = np.stack([math.cos(th) * y[:, 0] + math.sin(th) * y[:, 1], -math.sin(th) * y[:, 0] + math.cos(th) * y[:, 1]], 1)
    inside = (yb[:, 0] / 0.25) ** 2 + (yb[:, 1] / 0.15) ** 2 < 1.0
    assert np.array_equal(a == 1.0, inside)
    assert np.allclose(t.p[lm][inside, 0], 1.0) and np.allclose(t.p[lm][~inside, 1], 2e-3)
    # cells near the interface are at the maximum level
    assert (t.level[lm][inside] == 6).any()
    # honouring the key smears the interface
    tc2 = load_toml_case(_path("drop2d"), honour_diffuse_ic=True)
    a2 = tc2.case.tree.p[_leaves(tc2), 5]
    assert ((a2 > 0) & (a2 < 1)).any() and tc2.ignored == []


def test_bubble_jump_zone_and_periodic():
    tc = load_toml_case(_path("bubble_jump2d"))
    prm, t = tc.case.params, tc.case.tree
    lm = _leaves(tc)
    assert prm.sigma == 0.0 and prm.mu1 == 0.0
    we = load_toml_case(_write_text(open(_path("bubble_jump2d")).read().replace("L = 0.1", "L = 0.1\nWe = 0.02")))
    assert we.case.params.sigma == 1.0 / 0.02 and we.case.params.mu1 == 0.0  # We alone: tension, no viscosity
    with pytest.raises(ConfigError, match="needs We"):
        load_toml_case(_write_text(open(_path("bubble_jump2d")).read().replace("L = 0.1", "L = 0.1\nRe = 10.0")))
    assert list(prm.periodic) == [False, True]
    # jump: x > -1.5 takes value_pos, else value_neg, then the bubble's gas
    c, p = t.center[lm], t.p[lm]
    left = c[:, 0] <= -1.5
    assert np.allclose(p[left, 4], 7.0e7) and np.allclose(p[~left, 4], 1e5)
    bubble = np.hypot(c[:, 0] + 0.75, c[:, 1]) < 0.25
    assert np.allclose(p[bubble, 5], 0.0) and np.allclose(p[bubble, 1], 1.2) and np.allclose(p[bubble, 0], 0.0)
    assert np.allclose(p[~bubble & ~left, 0], 1000.0)
    # the zone (translated like the bubble: x0 = t + start) refines past the maximum level
    z = prm.zones[0]
    assert np.allclose(z.x0, [-2.0, -0.4, -1.0]) and np.allclose(z.x1, [-1.0, 0.4, 1.0]) and z.level == 7
    inz = z.contains(c)
    assert (t.level[lm][inz] == 7).all() and (t.level[lm][~inz] <= 5).all()
    # cells within one cell size of the jump refine to the maximum level
    near = np.abs(c[:, 0] + 1.5) < 0.5 ** t.level[lm] * 4.0
    assert (t.level[lm][near & ~inz] == 5).all()
    assert tc.case.tree.bcs[0].type == BcType.INFLOW_R


def test_navier_stokes_mach_reference():
    tc = load_toml_case(_path("channel_ns2d"))
    prm = tc.case.params
    mag = 0.3 * math.sqrt(1.4 * 101325.0 / 1.2)
    th = math.radians(2.0)
    assert np.allclose(tc.vel_ref, [mag * math.cos(th), mag * math.sin(th)], rtol=1e-15)
    mu = 1.2 * float(np.linalg.norm(tc.vel_ref)) * 0.5 / 150.0
    assert prm.ns_mu == mu and prm.ns_lambda == mu * 1005.0 / 0.72
    assert prm.max_dt == 1e-3 and tc.run.convergence_tol == 1e-6
    assert tc.case.tree.bcs[0].fade_in == 1e-3


def test_euler_mach_3d_direction(tmp_path):
    text = BASE.replace("domain_size = [1.0, 1.0]", "domain_size = [1.0, 1.0, 1.0]").replace(
        "vel = [0.5, 0.0]", "Ma = 0.5\nvel_angle = 10.0").replace(
        'min_refinement_level = 3', 'min_refinement_level = 2') + '[boundary_conditions.Z]\ntype = "periodic"\n'
    tc = load_toml_case(_write(tmp_path, text))
    mag = 0.5 * math.sqrt(1.4)
    th = math.radians(10.0)
    assert np.allclose(tc.vel_ref, [-mag * math.cos(th), 0.0, mag * math.sin(th)])  # model/euler.hpp:310-313


def test_multi_mach_uses_default_fluid_constants(tmp_path):
    text = open(_path("drop2d")).read().replace("vel = [0.0, 0.0]", "Ma = 0.1")
    tc = load_toml_case(_write(tmp_path, text))
    # alpha = 0: gas only, with the defaults gamma2 = 1.4, P2 = 0 (fluid_1 is read after the velocity)
    c = math.sqrt(1.4 * 1.0 / 2e-3)
    assert np.allclose(tc.vel_ref, [0.1 * c, 0.0])
    text2 = text.replace("alpha = 0.0", "alpha = 1.0")
    tc2 = load_toml_case(_write(tmp_path, text2, "c2"))
    c1 = math.sqrt(6.12 * (1.0 + 343000000.0) / 1.0)  # default gamma1, P1 although fluid_1 sets 5.5, 400
    assert np.allclose(tc2.vel_ref, [0.1 * c1, 0.0])


def test_geometry_support_and_rejections(tmp_path):
    drop = open(_path("drop2d")).read()
    with pytest.raises(ConfigError, match="Must define boundary condition"):
        load_toml_case(_write(tmp_path, drop.replace('type = "droplet"', 'type = "solid"')))
    with pytest.raises(NotImplementedError, match="STL"):
        load_toml_case(_write(tmp_path, drop.replace('shape = "ellipse"', 'path = "stl/x.stl"')))
    with pytest.raises(ConfigError):   # an airfoil needs camber, position and thickness
        load_toml_case(_write(tmp_path, drop.replace('shape = "ellipse"', 'shape = "naca_airfoil"')))
    with pytest.raises(ConfigError, match="Unknown shape type"):
        load_toml_case(_write(tmp_path, drop.replace('shape = "ellipse"', 'shape = "blob"')))
    # a diamond droplet: exact polygon signed distance
    dia = drop.replace('shape = "ellipse"', 'shape = "diamond"\nwidth = 0.6\nheight = 0.4').replace(
        "rotation = [0.0, 0.0, 30.0]", "rotation = [0.0, 0.0, 0.0]")
    tc = load_toml_case(_write(tmp_path, dia))
    t = tc.case.tree
    lm = _leaves(tc)
    y = t.center[lm] - [0.1, -0.05]
    inside = np.abs(y[:, 0]) / 0.3 + np.abs(y[:, 1]) / 0.2 < 1.0
    assert np.array_equal(t.p[lm, 5] == 1.0, inside)


def test_case_file_round_trip(tmp_path):
    for name in ("drop2d", "bubble_jump2d", "channel_ns2d"):
        tc = load_toml_case(_path(name))
        path = str(tmp_path / f"{name}.case")
        write_case(tc.case, path)
        back = read_case(path)
        assert np.array_equal(back.tree.p, tc.case.tree.p) and np.array_equal(back.tree.flags, tc.case.tree.flags)
        assert np.array_equal(back.params.param_vector(), tc.case.params.param_vector())
        assert len(back.params.zones) == len(tc.case.params.zones)


def _face_neighbours(t, nodes, act, periodic):
    """Same-level neighbour lookup (Domain::find) for every face of `nodes`: (n, 2D) node indices."""
    from dacti_b200.scene import _find

    class G:  # the tree's arrays under the names the lookup reads
        flags, level, center, children = t.flags, t.level, t.center, t.children

    D = t.center.shape[1]
    size = 4.0 * 0.5 ** t.level[nodes].astype(np.float64)
    out = np.zeros((nodes.size, 2 * D), np.int64)
    for d in range(D):
        for side_dir in range(2):
            ncen = t.center[nodes].copy()
            ncen[:, d] += (2.0 * side_dir - 1.0) * size
            out[:, 2 * d + side_dir] = _find(G, ncen, t.level[nodes], act, periodic)
    return out


def test_solid_cylinder_boundaries():
    tc = load_toml_case(_path("cylinder_ns2d"))
    t = tc.case.tree
    leaf = (t.flags & F_LEAF) != 0
    act = (t.flags & F_ACTIVE) != 0
    leaf[0] = False
    r = np.hypot(t.center[:, 0] + 0.8, t.center[:, 1])
    inbox = np.abs(t.center[:, 1]) < 1.0
    al, il = np.nonzero(leaf & act)[0], np.nonzero(leaf & ~act & inbox)[0]
    # scene.cpp:76-82: cells inside the solid are inactive, all others in the box active
    assert (r[il] < 0.2).all() and (r[al] > 0.2).all() and il.size > 0
    # object faces carry the no-slip condition, cells next to the solid are at the geometry level
    # and cannot coarsen (scene.cpp:118-138)
    obj = t.bc[al] >= 4
    walls = al[obj.any(axis=1)]
    assert walls.size > 0 and (t.level[walls] == 6).all()
    assert all(t.bcs[b].type == BcType.NOSLIP for b in np.unique(t.bc[al][obj]))
    from dacti_b200.models import F_CAN_UNSPLIT, F_IS_BOUNDARY
    assert ((t.flags[walls] & F_CAN_UNSPLIT) == 0).all() and ((t.flags[walls] & F_IS_BOUNDARY) != 0).all()
    # every face of an active leaf either has a condition or an active neighbour; faces with a
    # condition towards a cell of the box are paired with one on the other side (fix_boundary's last
    # pass, scene.cpp:316-334)
    act_box = np.array([4.0, 2.0])
    nb = _face_neighbours(t, al, act_box, [False, False])
    free = t.bc[al] < 0
    assert ((t.flags[nb[free]] & F_ACTIVE) != 0).all() and (nb[free] != 0).all()
    for f in range(4):
        has = (t.bc[al, f] >= 0) & (nb[:, f] != 0)
        opp = f ^ 1
        assert (t.bc[nb[has, f], opp] >= 0).all()
    # the wall normals are the circle's radial directions
    for i in walls[:8]:
        for f in np.nonzero(t.bc[i] >= 4)[0]:
            n = np.asarray(t.bcs[t.bc[i, f]].normal)
            radial = (t.center[i] - [-0.8, 0.0]) / r[i]
            assert np.allclose(n, radial, atol=1e-12)


def test_line_geometry_is_a_plate():
    """shape = "line" (geometry_data.hpp:75-93): a segment, here 0.8 long and turned by 10 degrees. No
    cell lies inside it. The faces it cuts carry its free-slip condition from both sides, and the cells
    there sit at the geometry level."""
    tc = load_toml_case(_path("plate_line2d"))
    t = tc.case.tree
    leaf = (t.flags & F_LEAF) != 0
    leaf[0] = False
    act = (t.flags & F_ACTIVE) != 0
    assert act[leaf].all()
    al = np.nonzero(leaf & act)[0]
    obj = t.bc[al] >= 4
    walls = al[obj.any(axis=1)]
    assert walls.size > 0
    assert all(t.bcs[b].type == BcType.FREESLIP for b in np.unique(t.bc[al][obj]))
    th = math.radians(10.0)
    x = t.center[walls]
    along = x[:, 0] * math.cos(th) + x[:, 1] * math.sin(th)
    across = -x[:, 0] * math.sin(th) + x[:, 1] * math.cos(th)
    size = 2.0 * 0.5 ** t.level[walls]
    assert (np.abs(across) < size).all() and (np.abs(along) <= 0.4 + size).all()
    assert (across > 0).any() and (across < 0).any()
    assert (t.level[walls] == 6).all()
    # the device builder keeps to polygons of 3 to 8 vertices; "auto" builds lines on the host
    auto = load_toml_case(_path("plate_line2d"), builder="auto")
    assert np.array_equal(auto.case.tree.bc, t.bc) and np.array_equal(auto.case.tree.level, t.level)


@pytest.mark.parametrize("shape,keys", [("naca_airfoil", 'camber = 0.02\nposition = 0.4\nthickness = 0.12'),
                                        ("Joukowski_airfoil", 'camber = 0.02\nthickness = 0.12')])
def test_airfoils_are_solid_polygons(shape, keys, tmp_path):
    """naca_airfoil and Joukowski_airfoil (scene/geometry.hpp:57-160), unit chord centred on the
    origin, turned by 10 degrees and made solid: the cells inside are inactive, the cells outside active,
    and the faces between them carry the wall."""
    text = open(_path("plate_line2d")).read().replace('shape = "line"\nlength = 0.8', f'shape = "{shape}"\n{keys}')
    tc = load_toml_case(_write(tmp_path, text))
    t = tc.case.tree
    obj = tc.objects[0]
    leaf = (t.flags & F_LEAF) != 0
    leaf[0] = False
    act = (t.flags & F_ACTIVE) != 0
    sd = obj.signed_distance(t.center)
    assert (sd[leaf & ~act] < 0).all() and (sd[leaf & act] > 0).all() and (leaf & ~act).any()
    th = math.radians(10.0)
    x = t.center[leaf & ~act]
    along = x[:, 0] * math.cos(th) + x[:, 1] * math.sin(th)
    across = -x[:, 0] * math.sin(th) + x[:, 1] * math.cos(th)
    assert (np.abs(along) <= 0.5).all() and (np.abs(across) < 0.09).all()
    al = np.nonzero(leaf & act)[0]
    walls = al[(t.bc[al] >= 4).any(axis=1)]
    assert walls.size > 0 and (t.level[walls] == 6).all()
