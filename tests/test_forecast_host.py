"""Regrid forecaster, host side: the CPU oracle of the network (gradients against central differences,
BF16 rounding) and the labels built from later solver states."""
import os
import sys

import numpy as np

from conftest import ROOT
from dacti_b200.casefile import Snapshot
from dacti_b200.forecast import best_threshold, region_labels, scores

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import forecast_mlp as ref  # noqa: E402


def test_oracle_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    n_in = 7
    p = rng.normal(0, 0.3, ref.n_params(n_in))
    x = rng.normal(size=(40, n_in))
    y = (rng.random(40) < 0.3).astype(float)
    loss, g = ref.loss_grad(p, x, y, 3.0)
    idx = rng.choice(p.size, 60, replace=False)
    for k in idx:
        e = np.zeros_like(p)
        e[k] = 1e-6
        num = (ref.loss_grad(p + e, x, y, 3.0)[0] - ref.loss_grad(p - e, x, y, 3.0)[0]) / 2e-6
        assert abs(num - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, num, g[k])
    # the loss is the weighted cross-entropy of the predicted probabilities
    q = ref.predict(p, x)
    assert np.isclose(loss, -(3.0 * y * np.log(q) + (1 - y) * np.log(1 - q)).sum())


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.14159265], np.float32)
    r = ref.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7  # above the tie rounds up
    assert r[3] == -2.5 and abs(r[4] - 3.140625) < 1e-12


def _snap(levels, centers, errors):
    n = len(levels)
    z = np.zeros(n)
    c = np.asarray(centers, float)
    return Snapshot(2, 4, 0, 0, 0, n, 0.0, 0.0, 0.0, np.asarray(levels, np.int32), np.zeros(n, np.int32), c, z,
                    np.ones((n, 4)), np.ones((n, 4)), np.asarray(errors, float), z, z)


def test_region_labels():
    side = 1.0
    # now: four level-1 leaves (quadrants of the unit box centred at the origin)
    q = [(-0.25, -0.25), (0.25, -0.25), (-0.25, 0.25), (0.25, 0.25)]
    now = _snap([1, 1, 1, 1], q, [0.0, 0.0, 0.0, 0.0])
    # future: quadrant 0 refined (four level-2 leaves), quadrant 1 flagged, 2 and 3 quiet
    kids = [(-0.375, -0.375), (-0.125, -0.375), (-0.375, -0.125), (-0.125, -0.125)]
    fut = _snap([2, 2, 2, 2, 1, 1, 1], kids + q[1:], [0, 0, 0, 0, 0.5, 0.0, 0.0])
    lab = region_labels(now, fut, side, max_err=0.1)
    assert lab.tolist() == [True, True, False, False]
    # a fine leaf now inside a coarse flagged future leaf is positive; inside a quiet one negative
    now2 = _snap([2, 2], [(0.125, -0.125), (0.125, 0.375)], [0.0, 0.0])
    assert region_labels(now2, fut, side, max_err=0.1).tolist() == [True, False]


def test_scores_and_threshold():
    truth = np.array([1, 1, 0, 0, 1], bool)
    s = scores(np.array([1, 0, 0, 1, 1], bool), truth)
    assert s["tp"] == 2 and s["fp"] == 1 and s["fn"] == 1 and np.isclose(s["f1"], 2 / 3)
    prob = np.array([0.9, 0.8, 0.2, 0.1, 0.7])
    assert scores(prob >= best_threshold(prob, truth), truth)["f1"] == 1.0
