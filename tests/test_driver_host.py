"""The default_driver loop (driver/default_driver.hpp:77-217) on the host, over a stand-in solver that
needs no GPU: frame cadence, the observables CSV, the steady-state stop and the NaN break."""
import csv

import numpy as np

from dacti_b200.casefile import Snapshot
from dacti_b200.driver import DefaultDriver, Totals
from dacti_b200.io import read_vtu_arrays


class FakeSolver:
    """integrate() advances by a fixed dt; the state decays towards a steady value, and a NaN can be
    reported at a chosen step."""

    side_length = 1.0

    def __init__(self, dt=0.01, decay=0.5, nan_at=None):
        self.dt, self.decay, self.nan_at, self.calls, self.signals = dt, decay, nan_at, 0, []
        lv = np.array([1, 1, 1, 1], np.int32)
        c = np.array([[-0.25, -0.25], [0.25, -0.25], [-0.25, 0.25], [0.25, 0.25]])
        self.u = np.tile([1.0, 0.0, 0.0, 2.5], (4, 1))
        self.u[0, 0] = 2.0
        self._lv, self._c = lv, c

    def integrate(self, signal=True):
        self.calls += 1
        self.signals.append(signal)
        self.u[0, 0] = 1.0 + (self.u[0, 0] - 1.0) * self.decay
        return self.dt, self.nan_at is not None and self.calls >= self.nan_at

    def active_cells(self):
        n = 4
        return Snapshot(2, 4, self.calls, 0, 5, n, 0.0, self.dt, 0.0, self._lv, np.zeros(n, np.int32), self._c,
                        np.zeros(n), self.u.copy(), self.u.copy(), np.zeros(n), np.zeros(n), np.zeros(n))

    def active_slopes(self):
        return np.zeros((4, 2, 4))


def _rows(path):
    rows = list(csv.reader(open(path)))
    return rows[0], [[float(x) for x in r] for r in rows[1:]]


def test_frame_cadence_and_csv(tmp_path):
    s = FakeSolver(dt=0.01, decay=1.0)
    res = DefaultDriver(s, "f", str(tmp_path), end_time=0.1, io_interval=0.025, observers=[Totals(4)],
                        signal_time=0.03).run()
    # 10 steps of 0.01 (the last one may land a rounding step short of 0.1 and take an 11th)
    assert res["steps"] in (10, 11) and res["time"] >= 0.1 - 1e-12
    head, rows = _rows(tmp_path / "f_observables.csv")
    assert head == ["time", "frame", "step", "n_cells", "u_0", "u_1", "u_2", "u_3"]
    # a frame whenever the time advanced by at least io_interval since the last one
    times = [r[0] for r in rows]
    assert all(b - a >= 0.025 - 1e-12 for a, b in zip([0.0] + times[:-1], times))
    assert [int(r[1]) for r in rows] == list(range(1, len(rows) + 1))
    assert all(r[3] == 4 for r in rows)
    assert np.allclose([r[4] for r in rows], (2.0 + 3.0) * 0.25)
    # signal = time > signal_time, evaluated before each step
    t = np.arange(len(s.signals)) * 0.01
    assert s.signals == [bool(x > 0.03) for x in t]
    for f in range(res["frames"] + 1):
        assert read_vtu_arrays(str(tmp_path / f"f_{f:04d}.vtu"))["types"].size == 4


def test_steady_state_stop(tmp_path):
    s = FakeSolver(dt=0.01, decay=0.5)
    res = DefaultDriver(s, "c", str(tmp_path), end_time=10.0, io_interval=1.0, observers=[Totals(4)],
                        convergence_tol=1e-3, write_frames=False).run()
    assert res["converged"] and res["time"] < 10.0
    head, rows = _rows(tmp_path / "c_observables.csv")
    # every step appends a row while a tolerance is set; the converged step also writes a frame row
    assert len(rows) >= res["steps"]
    mass = np.array([r[4] for r in rows])
    assert abs(mass[-1] - 0.25 * 4.0) < 1e-3 * 0.01 * 4 + 1e-12


def test_nan_break_writes_its_frame(tmp_path):
    s = FakeSolver(dt=0.01, decay=1.0, nan_at=3)
    res = DefaultDriver(s, "n", str(tmp_path), end_time=1.0, io_interval=0.5, observers=[Totals(4)]).run()
    assert res["force_break"] and s.calls == 3
    assert res["frames"] == 1  # the NaN step forces a frame before the loop ends
    assert (tmp_path / "n_0001.vtu").exists()


class FakeTreeSolver(FakeSolver):
    """FakeSolver whose four cells are the children of one root, for the HTG writer."""

    class params:
        active_size = (1.0, 1.0)

    def tree_nodes(self):
        from dacti_b200.htg import NodeTable
        n = 6
        children = np.zeros((n, 4), np.int32)
        children[1] = [2, 3, 4, 5]
        flags = np.array([0, 2, 3, 3, 3, 3], np.uint32)
        p = np.zeros((n, 4))
        p[2:] = self.u
        return NodeTable(2, np.array([0, 0, 1, 1, 1, 1], np.int32), children, np.array([0, 0, 1, 1, 1, 1], np.int32),
                         flags, p, np.zeros((n, 4)))


def test_htg_frames(tmp_path):
    from dacti_b200.htg import read_htg
    s = FakeTreeSolver(dt=0.01, decay=0.5)
    res = DefaultDriver(s, "h", str(tmp_path), end_time=0.05, io_interval=0.02, observers=[Totals(4)],
                        writer="htg").run()
    assert res["frames"] >= 2
    for f in range(res["frames"] + 1):
        a = read_htg(str(tmp_path / f"h_{f:04d}.htg"))
        assert a["NbVerticesByLevel"].tolist() == [1, 4]
        assert a["Descriptor"].tolist() == [True]
    last = read_htg(str(tmp_path / f"h_{res['frames']:04d}.htg"))
    # the leaves carry the state of a step (the decaying first cell, the other three at 1); the root
    # vertex gets no value
    assert 1.0 < last["p_0"][1] < 2.0 and np.all(last["p_0"][2:] == 1.0) and last["p_0"][0] == 0.0
    assert not (tmp_path / "h_0000.vtu").exists()
    import pytest
    with pytest.raises(ValueError):
        DefaultDriver(s, "h", str(tmp_path), writer="xdmf")
