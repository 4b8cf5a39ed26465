"""The default_driver loop over the GPU solver: frames, observables CSV and VTU files, and the
conservation the Totals observer reports on a periodic case."""
import csv
import os

import numpy as np
import pytest

from dacti_b200 import cases
from dacti_b200.driver import DefaultDriver, Totals
from dacti_b200.io import read_vtu_arrays
from dacti_b200.solver import Solver

pytestmark = pytest.mark.gpu


def test_driver_writes_frames_and_observables(tmp_path):
    case = cases.periodic_blob(base_level=4, levels=2)
    s = Solver(case)
    d = DefaultDriver(s, "blob", str(tmp_path), end_time=0.1, io_interval=0.03, observers=[Totals(4)])
    res = d.run()
    assert res["time"] >= 0.1 and not res["force_break"] and res["frames"] >= 3
    rows = list(csv.reader(open(tmp_path / "blob_observables.csv")))
    assert rows[0] == ["time", "frame", "step", "n_cells", "u_0", "u_1", "u_2", "u_3"]
    assert len(rows) == 1 + res["frames"]
    mass = np.array([float(r[4]) for r in rows[1:]])
    assert np.allclose(mass, mass[0], rtol=1e-12)  # periodic: mass is conserved
    for f in range(res["frames"] + 1):
        a = read_vtu_arrays(str(tmp_path / f"blob_{f:04d}.vtu"))
        assert a["types"].size == a["Points"].shape[0] // 8
    last = read_vtu_arrays(str(tmp_path / f"blob_{res['frames']:04d}.vtu"))
    assert last["types"].size == s.n_active_cells()
    s.close()
