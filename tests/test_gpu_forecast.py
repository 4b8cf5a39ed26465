"""Regrid forecaster on the GPU: the network's kernels against the CPU oracle (loss and gradient of
the FP32 master weights, predictions with BF16 weights), training, the solver's feature kernel, and what
the trained network gains over the method without it on a held-out cylinder-flow run."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from dacti_b200 import cases
from dacti_b200.forecast import Mlp, collect, run_with_forecast, scores, train_forecaster
from dacti_b200.solver import Solver

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import forecast_mlp as ref  # noqa: E402

pytestmark = pytest.mark.gpu


def test_loss_gradient_matches_oracle():
    rng = np.random.default_rng(1)
    n_in = 15
    net = Mlp(n_in, seed=3)
    p = net.params
    assert p.size == ref.n_params(n_in)
    x = rng.normal(size=(700, n_in)).astype(np.float32)
    y = (rng.random(700) < 0.25).astype(np.float32)
    loss, g = net.loss_grad(x, y, pos_weight=3.0)
    rl, rg = ref.loss_grad(p.astype(np.float64), x, y, 3.0)
    assert abs(loss - rl) <= 1e-5 * abs(rl)
    scale = np.abs(rg).max()
    assert np.abs(g - rg).max() <= 1e-4 * scale, np.abs(g - rg).max() / scale
    net.close()


def test_predictions_use_bf16_weights():
    rng = np.random.default_rng(2)
    net = Mlp(20, seed=5)
    p = rng.normal(0, 0.2, net.n_params).astype(np.float32)
    net.params = p
    assert np.array_equal(net.params, p)
    x = rng.normal(size=(513, 20)).astype(np.float32)
    got = net.predict(x)
    want = ref.predict(ref.bf16(p), x)
    assert np.abs(got - want).max() <= 2e-5
    # the FP32 master weights would give a visibly different answer
    assert np.abs(ref.predict(p.astype(np.float64), x) - want).max() > 1e-4
    net.close()


def test_training_separates_a_toy_problem():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(8000, 6)).astype(np.float32)
    y = ((x[:, 0] + 0.5 * x[:, 1] * x[:, 2]) > 0.3).astype(np.float32)
    net = Mlp(6, seed=9)
    first = net.loss_grad(x, y)[0] / y.size
    last = net.train(x, y, epochs=15, batch=256, lr=3e-3)
    assert last < 0.5 * first and last < 0.25
    acc = ((net.predict(x) >= 0.5) == (y > 0.5)).mean()
    assert acc > 0.93
    net.close()


def test_features_of_the_solver():
    s = Solver(cases.cylinder_ns(base_level=5, levels=2))
    for _ in range(2):
        s.integrate()
    f = s.forecast_features()
    snap = s.active_cells()
    assert f.shape == (snap.n, 15) and np.isfinite(f).all()
    assert np.allclose(f[:, 3], snap.tree_level / 16.0)
    max_err = s.params.error_threshold[1]
    assert np.allclose(f[:, 4], np.log1p(np.maximum(snap.error, 0.0) / max_err), rtol=1e-6, atol=1e-7)
    # velocity over (|v| + c): the inflow moves along +x at Mach ~0.3
    assert np.median(f[:, 5]) > 0.15 and np.abs(f[:, 6]).max() < 1.0
    # density-gradient features: zero-gradient regions give 0, compressed values stay moderate
    assert (f[:, 0] >= 0).all() and f[:, 0].max() < 12
    s.close()


def _run(seed, steps=20, horizon=8):
    mach = float(np.random.default_rng(seed).uniform(0.2, 0.4))
    return collect(lambda: cases.cylinder_ns(mach=mach, base_level=5, levels=3), steps, horizon)


def test_forecaster_beats_persistence_on_a_held_out_run():
    train = [_run(s) for s in (11, 12, 13)]
    test = _run(21)
    net, cut, loss = train_forecaster(train, n_in=15, epochs=30)
    pred = net.predict(test.x) >= cut
    truth = test.y.astype(bool)
    mlp, base = scores(pred, truth), scores(test.persistence, truth)
    print("forecaster", mlp, "persistence", base, "cut", cut, "loss", loss, "samples", truth.size,
          "positive rate", truth.mean())
    assert truth.any() and (~truth).any()
    assert mlp["f1"] > base["f1"] + 0.05
    assert mlp["recall"] > base["recall"]
    net.close()


def _cyl():
    return cases.cylinder_ns(mach=0.3, base_level=5, levels=3)


def test_regrid_controls_default_to_the_reference():
    a, b = Solver(_cyl()), Solver(_cyl())
    b.set_coarsen_interval(1)
    b.set_hold(np.zeros(b.n_active_cells(), np.uint8))
    for _ in range(3):
        a.integrate()
        b.integrate()
    sa, sb = a.active_cells(), b.active_cells()
    assert np.array_equal(sa.tree_level, sb.tree_level) and np.array_equal(sa.u, sb.u)
    a.close(), b.close()


def _coarsened(before, after, side=40.0):
    """Leaves of `after` coarser than the leaves of `before` at their place."""
    from dacti_b200.casefile import cell_coords
    from dacti_b200.forecast import _keys

    kb = set(_keys(before.tree_level, cell_coords(before.center, before.tree_level, side)).tolist())
    la = after.tree_level.astype(np.int64)
    ca = cell_coords(after.center, la, side)
    found = np.zeros(la.size, bool)
    for l in range(int(la.max()) + 1):
        m = la >= l
        anc = _keys(np.full(m.sum(), l), ca[m] >> (la[m] - l)[:, None])
        found[np.nonzero(m)[0][np.isin(anc, np.fromiter(kb, np.uint64))]] = True
    return int((~found).sum())


def test_held_cells_never_coarsen():
    free, held = Solver(_cyl()), Solver(_cyl())
    for _ in range(6):  # the start-up transient refines around the cylinder and the wake
        free.integrate()
        held.integrate()
    f6, h6 = free.active_cells(), held.active_cells()
    held.set_hold(np.ones(held.n_active_cells(), np.uint8))
    for _ in range(6):
        free.integrate()
        held.integrate()
    # the free run coarsens some of the step-6 cells again; none of the held ones is (cells created
    # after the hold are not held)
    assert _coarsened(f6, free.active_cells()) > 0
    assert _coarsened(h6, held.active_cells()) == 0
    # coarsening skipped on global steps that are not multiples of the interval
    free.set_coarsen_interval(8)
    u0 = free.stats().n_unsplits
    free.integrate()  # global step 12
    free.integrate()  # global step 13
    assert free.stats().n_unsplits == u0
    free.close(), held.close()


def test_forecast_driven_regrid_against_plain():
    from dacti_b200.accuracy import density_rel_l1

    train = [_run(s) for s in (11, 12, 13)]
    net, cut, _ = train_forecaster(train, n_in=15, epochs=30)
    plain, fc = Solver(_cyl()), Solver(_cyl())
    for _ in range(16):
        plain.integrate()
    res = run_with_forecast(fc, net, cut, steps=16, interval=8, coarsen_every=1)
    sp = plain.stats()
    err = density_rel_l1(plain.active_cells(), fc.active_cells(), 40.0, (40.0, 20.0), 8, 1)
    print("plain splits", sp.n_splits, "unsplits", sp.n_unsplits, "updates", sp.cell_updates,
          "| forecast", res, "| density rel-L1 vs plain", err)
    assert not res["force_break"]
    # held cells are never coarsened, so the regrid does less split/unsplit churn
    assert res["unsplits"] < sp.n_unsplits
    assert res["splits"] + res["unsplits"] < sp.n_splits + sp.n_unsplits
    assert err < 5e-3
    plain.close(), fc.close()
    net.close()
