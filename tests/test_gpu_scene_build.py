"""The initial tree built on the GPU (dg_build_tree) against the host builder: the same nodes in the
same order, the same flags, boundary ids and centres bit for bit, and the same primitive states (the
smeared volume fraction within a few ulps: CUDA's tanh against numpy's)."""
import os
import time

import numpy as np
import pytest

from conftest import GOLDEN
from dacti_b200 import cases
from dacti_b200.scene import build_tree
from dacti_b200.scene_gpu import build_tree_device
from dacti_b200.toml_case import load_toml_case

pytestmark = pytest.mark.gpu


def _bc_specs(t):
    """Each face's boundary as (type, state, normal), None without one: the boundary table's numbering
    is free."""
    keys = [(int(b.type), tuple(b.p_in), tuple(b.normal), float(b.fade_in)) for b in t.bcs]
    return [[keys[k] if k >= 0 else None for k in row] for row in t.bc.tolist()]


def _same(a, b):
    for name in ("parent", "children", "level", "flags", "center"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape and np.array_equal(x, y), name
    assert np.allclose(a.p, b.p, rtol=1e-14, atol=1e-14 * np.abs(a.p).max())
    assert _bc_specs(a) == _bc_specs(b)


@pytest.mark.parametrize("dims,base,levels", [(2, 5, 3), (3, 4, 2)])
def test_shock_drop_tree(dims, base, levels):
    spec, _ = cases.shock_drop_spec(dims=dims, base_level=base, levels=levels)
    _same(build_tree(spec), build_tree_device(spec))


@pytest.mark.parametrize("name,diffuse", [("drop2d", False), ("drop2d", True), ("bubble_jump2d", False),
                                          ("channel_ns2d", False)])
def test_toml_scene_tree(name, diffuse):
    tc = load_toml_case(os.path.join(GOLDEN, "toml", f"{name}.toml"), honour_diffuse_ic=diffuse)
    _same(tc.case.tree, build_tree_device(tc.spec))


def test_solid_objects():
    # object faces, fix_boundary and the one-sided boundary drop on the device
    tc = load_toml_case(os.path.join(GOLDEN, "toml", "cylinder_ns2d.toml"))
    dev = build_tree_device(tc.spec)
    _same(tc.case.tree, dev)
    from dacti_b200.models import F_ACTIVE, F_IS_BOUNDARY, F_LEAF
    assert ((dev.flags & F_IS_BOUNDARY) != 0).any() and ((dev.flags & (F_LEAF | F_ACTIVE)) == F_LEAF).any()
    spec, _ = cases.cylinder_ns_spec(base_level=5, levels=3)
    _same(build_tree(spec), build_tree_device(spec))


@pytest.mark.parametrize("shape", ['shape = "diamond"\nwidth = 0.4\nheight = 0.3',
                                   'shape = "triangle"\nv1 = [0.2, 0.0]\nv2 = [-0.15, 0.18]\nv3 = [-0.1, -0.2]'])
def test_polygon_solids(tmp_path, shape):
    text = open(os.path.join(GOLDEN, "toml", "cylinder_ns2d.toml")).read().replace(
        'shape = "circle"\nradius = 0.2', shape)
    path = tmp_path / "poly.toml"
    path.write_text(text)
    tc = load_toml_case(str(path))
    _same(tc.case.tree, build_tree_device(tc.spec))


def test_full_size_shock_drop_build_time():
    spec, _ = cases.shock_drop_spec()  # 64 x 32 x 32 base, +4 levels
    build_tree_device(cases.shock_drop_spec(base_level=3, levels=1)[0])  # context and code warm
    t0 = time.perf_counter()
    dev = build_tree_device(spec)
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    host = build_tree(spec)
    t_host = time.perf_counter() - t0
    print(f"shock-drop 3D tree: {dev.n_nodes} nodes, device {t_dev:.3f} s (with host copies), host {t_host:.2f} s")
    _same(host, dev)


def test_toml_loader_device_builder():
    for name in ("bubble_jump2d", "cylinder_ns2d"):
        host = load_toml_case(os.path.join(GOLDEN, "toml", f"{name}.toml"))
        dev = load_toml_case(os.path.join(GOLDEN, "toml", f"{name}.toml"), builder="device")
        _same(host.case.tree, dev.case.tree)
