"""HTG frames from the device tree (dg_read_tree) against DACTI's own integrator after the same steps.

The reference runner dumps Integrator::get_nodes() (--nodes); the oracle replays DACTI's htg_writer on
that table (oracle/htg_writer_ref.py). The device's node pool, read back with dg_read_tree and walked
by dacti_b200/htg.py, must give the same hyper tree (descriptor, vertices per level, mask) and the
same values at every written vertex:
- acti_level: exact;
- p: exact after construction, rel-L1 <= 1e-10 per component after steps (the parity bar);
- error, max_dt, cfl: exact after construction, close after steps.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, run_reference
from dacti_b200.casefile import read_case
from dacti_b200.driver import DefaultDriver, Totals
from dacti_b200.htg import hyper_tree, read_htg
from dacti_b200.solver import Solver
from oracle.htg_writer_ref import read_nodes, reference_htg

pytestmark = pytest.mark.gpu


def _ref_arrays(path):
    d = read_nodes(path)
    desc, per_depth, mask, data = reference_htg(d["dims"], d["parent"], d["children"], d["level"], d["flags"], d["p"],
                                                d["meta"], d["root"])
    written = np.array([v is not None for v in data["p_0"]])
    vals = {k: np.array([0.0 if x is None else x for x in v]) for k, v in data.items()}
    return np.array(desc, bool), np.array(per_depth), np.array(mask, bool), written, vals, d["E"]


@pytest.mark.parametrize("name,steps", [("euler2", 6), ("multi2", 4), ("euler3", 2)])
def test_device_tree_matches_reference_nodes(name, steps, tmp_path):
    case = read_case(os.path.join(GOLDEN, f"{name}.case"))
    run_reference(os.path.join(GOLDEN, f"{name}.case"), str(tmp_path / name), steps, [0, steps], extra=("--nodes",))
    s = Solver(case)
    try:
        for k in (0, steps):
            if k > 0:
                for _ in range(steps):
                    _, fb = s.integrate()
                    assert not fb
            ht = hyper_tree(s.tree_nodes(), case.params.active_size[0])
            desc, per_depth, mask, written, vals, E = _ref_arrays(str(tmp_path / f"{name}_{k}.nodes"))
            assert np.array_equal(ht.vertices_per_level, per_depth)
            assert np.array_equal(ht.descriptor, desc)
            assert np.array_equal(ht.mask, mask)
            w = written
            assert np.array_equal(ht.cell_data["acti_level"][w], vals["acti_level"][w])
            dev = {}
            for q in range(E):
                a, b = ht.cell_data[f"p_{q}"][w], vals[f"p_{q}"][w]
                if k == 0:
                    assert np.array_equal(a, b), q
                else:
                    rel = np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)
                    assert rel <= 1e-10, (q, rel)
            for nm in ("error", "max_dt", "cfl"):
                a, b = ht.cell_data[nm][w], vals[nm][w]
                dev[nm] = float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))) if a.size else 0.0
                if k == 0:
                    assert np.array_equal(a, b), nm
                else:
                    scale = np.abs(b).max() if b.size else 0.0
                    assert np.all(np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-6 * scale), nm
            print(f"{name} step {k}: {ht.n_vertices} vertices, {int(ht.mask.sum())} masked, "
                  f"max rel dev error {dev['error']:.2e} max_dt {dev['max_dt']:.2e} cfl {dev['cfl']:.2e}")
    finally:
        s.close()


def test_driver_writes_htg_frames(tmp_path):
    case = read_case(os.path.join(GOLDEN, "euler2.case"))
    s = Solver(case)
    try:
        res = DefaultDriver(s, "e", str(tmp_path), end_time=1e9, io_interval=0.0, observers=[Totals(4)],
                            writer="htg", max_steps=2).run()
        assert res["steps"] == 2
        a = read_htg(str(tmp_path / "e_0002.htg"))
        shown = (a["p_0"] != 0) & ~a["Mask"]
        assert int(shown.sum()) == s.n_active_cells()
        assert a["NumberOfVertices"][0] == a["NbVerticesByLevel"].sum()
    finally:
        s.close()
