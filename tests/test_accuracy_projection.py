"""Conservative projection used to compare solutions on different adaptive meshes (no GPU)."""
import os

import numpy as np

from conftest import GOLDEN
from dacti_b200.accuracy import density_rel_l1, project_uniform
from dacti_b200.casefile import read_case, read_snapshot


def test_projection_conserves_totals_and_is_zero_against_itself():
    case = read_case(os.path.join(GOLDEN, "multi2.case"))
    snap = read_snapshot(os.path.join(GOLDEN, "multi2_4.snap"))
    side, act = case.params.side_length, case.params.active_size
    for level in (3, 4, 6):
        out = project_uniform(snap, side, act, level)
        h = side / (1 << level)
        vol_leaf = (side * 0.5 ** snap.tree_level.astype(float)) ** 2
        scale = (np.abs(snap.u) * vol_leaf[:, None]).sum(axis=0)
        assert np.all(np.abs(out.sum(axis=0) * h * h - (snap.u * vol_leaf[:, None]).sum(axis=0)) <= 1e-12 * scale)
        assert density_rel_l1(snap, snap, side, act, level, 2) == 0.0


def test_projection_detects_a_perturbation():
    case = read_case(os.path.join(GOLDEN, "euler2.case"))
    a = read_snapshot(os.path.join(GOLDEN, "euler2_6.snap"))
    b = read_snapshot(os.path.join(GOLDEN, "euler2_6.snap"))
    b.u[:, 0] *= 1 + 1e-6
    err = density_rel_l1(b, a, case.params.side_length, case.params.active_size, 3, 0)
    assert abs(err - 1e-6) < 1e-9
