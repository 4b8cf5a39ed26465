"""VTU output (driver/io/vtu_writer.hpp restated): voxel geometry, vertex values from the linear
reconstruction, cell data; decoded back from the written file."""
import numpy as np

from dacti_b200.casefile import Snapshot
from dacti_b200.io import read_vtu_arrays, voxel_points, write_vtu


def _snap(dims=2, E=4, n=5, seed=0):
    rng = np.random.default_rng(seed)
    lv = rng.integers(2, 5, n).astype(np.int32)
    return Snapshot(dims, E, 0, 0, 0, n, 0.0, 0.0, 0.0, lv, rng.integers(0, 3, n).astype(np.int32),
                    rng.uniform(-0.4, 0.4, (n, dims)), np.zeros(n), rng.uniform(1, 2, (n, E)),
                    rng.uniform(1, 2, (n, E)), rng.uniform(0, 1, n), rng.uniform(0, 1, n), rng.uniform(0, 1, n))


def test_vtu_round_trip(tmp_path):
    snap = _snap()
    slopes = np.random.default_rng(1).normal(size=(snap.n, snap.dims, snap.E))
    path = str(tmp_path / "f.vtu")
    write_vtu(path, snap, slopes, 1.0, fields={"extra": np.arange(snap.n, dtype=np.float64)})
    a = read_vtu_arrays(path)
    assert a["Points"].shape == (8 * snap.n, 3)
    assert np.array_equal(a["types"], np.full(snap.n, 11, np.uint8))
    assert np.array_equal(a["offsets"], 8 * np.arange(1, snap.n + 1))
    assert np.array_equal(a["error"], snap.error) and np.array_equal(a["acti_level"], snap.acti_level)
    assert np.array_equal(a["extra"], np.arange(snap.n))
    pts = voxel_points(snap, 1.0)
    size = 0.5 ** snap.tree_level
    # vertex j of a cell sits at centre + size/2 * quadrant(j); 2D cells get a z extent of 0.01
    assert np.allclose(pts[:, 7, :2] - pts[:, 0, :2], size[:, None])
    assert np.allclose(pts[:, 7, 2] - pts[:, 0, 2], 0.01)
    # vertex values p + slope (x - c): their mean over the 8 vertices is p
    for q in range(snap.E):
        v = a[f"p_{q}"].reshape(snap.n, 8)
        assert np.allclose(v.mean(axis=1), snap.p[:, q])
        x = pts[:, 0, :2] - snap.center
        assert np.allclose(v[:, 0], snap.p[:, q] + (slopes[:, :, q] * x).sum(axis=1))
