"""The stage implementation choices (dg_set_options) give the same results bit for bit.

The ordered list rebuild and the tiled face sums change only the order of list positions and which
thread evaluates a face, never an operand or the order of a sum; each case runs every combination
of the two choices for several global steps and compares the active cells, their ACTI levels, the
conserved state and the step counters exactly.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from dacti_b200 import cases
from dacti_b200.casefile import read_case
from dacti_b200.solver import OPT_FACE_TILES, OPT_ORDERED_LISTS, Solver

pytestmark = pytest.mark.gpu

COMBOS = (0, OPT_ORDERED_LISTS, OPT_FACE_TILES, OPT_ORDERED_LISTS | OPT_FACE_TILES)


def _run(case, options, steps, form="fp64"):
    s = Solver(case)
    s.set_form(form)
    s.set_options(options)
    dts = []
    for _ in range(steps):
        gdt, fb = s.integrate()
        assert not fb
        dts.append(gdt)
    snap = s.active_cells()
    st = s.stats()
    s.close()
    return snap, dts, (st.cell_updates, st.n_splits, st.n_unsplits, st.n_substeps, st.tree_size)


def _sorted(snap, side):
    from dacti_b200.parity import _keys
    order = np.argsort(_keys(snap, side))
    return snap.u[order], snap.acti_level[order], snap.tree_level[order], _keys(snap, side)[order]


def _check_same(case, steps, form="fp64"):
    side = case.params.side_length
    base = None
    for opt in COMBOS:
        snap, dts, counters = _run(case, opt, steps, form)
        got = (_sorted(snap, side), dts, counters)
        if base is None:
            base = got
            continue
        (u0, a0, l0, k0), d0, c0 = base
        (u1, a1, l1, k1), d1, c1 = got
        assert np.array_equal(k0, k1), f"options {opt}: cell sets differ"
        assert np.array_equal(a0, a1) and np.array_equal(l0, l1), f"options {opt}: levels differ"
        assert np.array_equal(u0.view(np.int64), u1.view(np.int64)), f"options {opt}: state differs"
        assert d0 == d1 and c0 == c1, f"options {opt}: {d1} {c1} against {d0} {c0}"


@pytest.mark.parametrize("name,steps", [("multi3", 2), ("multi2", 4), ("ns3", 4), ("euler2_walls", 5),
                                        ("multi2_visc", 4), ("euler2_periodic", 4)])
def test_options_bitwise_on_golden_cases(name, steps):
    _check_same(read_case(os.path.join(GOLDEN, f"{name}.case")), steps)


def test_options_bitwise_on_shock_drop():
    """The benchmark's scene at 32 x 16 x 16 + 3 levels: hanging faces in three directions, receivers of
    slower clusters, splits and coarsenings in every substep, lists rebuilt at every level."""
    _check_same(cases.shock_drop(base_level=5, levels=3), 2)


def test_options_bitwise_mixed_form():
    _check_same(cases.shock_drop(base_level=4, levels=2), 2, form="mixed")
