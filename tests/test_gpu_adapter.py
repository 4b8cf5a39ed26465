"""The C++ adapter include/dacti_gpu/integrator.hpp is a drop-in for the reference's Integrator.

oracle/_ref/dacti_adapter_check holds, in one process, the reference's
dacti::integrator::Integrator (integrator/integrator.hpp:14-225, compiled from its own headers) and
dacti::gpu::Integrator over the GPU library, both built from the same Scene and Config, and drives
them with the same calls a DACTI driver makes (integrate with a substep hook, n_active_cells,
for_each_active_cell, global_dt). After construction and after every global step it compares the
hook sequence, force_break, global_dt, the active cell set with ACTI levels, the conserved state
(relative L1 <= 1e-10), and the slopes and gradients the adapter's nodes carry (relative L1 <= 1e-8;
gradients where the case has viscous or conduction terms), printing one JSON line per step. For the
multiphase cases DACTI's own DropEnergy observer (driver/observer/drop_energy.hpp), compiled unchanged
into the same binary, runs on both integrators after the last step. After the last step both
integrators' get_nodes() trees, the input of DACTI's htg_writer, are dumped and compared.
"""
import json
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT

CHECK = os.path.join(ROOT, "oracle", "_ref", "dacti_adapter_check")

CASES = [("euler2", 4), ("ns2", 4), ("multi2", 3), ("multi3", 2), ("euler3", 4), ("ns3", 4), ("euler2_periodic", 4), ("euler2_walls", 6),
         ("euler2_open_a", 6), ("euler2_lim2", 4), ("euler2_lim5", 4), ("multi2_tension_run", 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,steps", CASES)
def test_adapter_matches_reference_integrator(name, steps, tmp_path):
    if not os.path.exists(CHECK):
        pytest.fail("oracle/_ref/dacti_adapter_check is not built (make -C oracle after building the library)")
    r = subprocess.run([CHECK, os.path.join(GOLDEN, f"{name}.case"), str(tmp_path / name), str(steps),
                        "--adapter-check", "--nodes"], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert r.returncode == 0, r.stdout + r.stderr
    assert len(lines) == steps + 1
    for rec in lines:
        assert rec["hooks_equal"] and rec["force_break_equal"] and rec["cells_equal"], rec
        assert rec["global_dt_equal"] and rec["n_ref"] == rec["n_gpu"] and rec["rel_l1_u"] <= 1e-10, rec
        # slopes (read by Cell::get_p) and gradients (read by DropEnergy) as the adapter hands them out
        assert rec["rel_l1_slope"] <= 1e-8 and rec["rel_l1_grad"] <= 1e-8, rec
    # DACTI's DropEnergy observer, compiled unchanged, reads the same kinetic and total energy from both
    de = [json.loads(x[len("DROP_ENERGY "):]) for x in r.stdout.splitlines() if x.startswith("DROP_ENERGY ")]
    if name.startswith("multi"):
        assert len(de) == 1
        for a, b in zip(de[0]["ref"], de[0]["gpu"]):
            assert abs(a - b) <= 1e-8 * max(abs(a), 1e-300), de
    _same_hyper_tree(str(tmp_path / f"{name}_ref.nodes"), str(tmp_path / f"{name}_adapter.nodes"))


def _same_hyper_tree(ref_path, adapter_path):
    """The adapter's get_nodes() (the whole device tree, renumbered from root slot 1) gives DACTI's
    htg_writer the hyper tree that the reference integrator's get_nodes() gives it: same subdivisions,
    mask and ACTI levels, p within the parity bar, max_dt and cfl within 1e-12, the error estimate
    within 1e-6 of its largest value."""
    import numpy as np
    from oracle.htg_writer_ref import read_nodes, reference_htg

    trees = []
    for path in (ref_path, adapter_path):
        d = read_nodes(path)
        trees.append(reference_htg(d["dims"], d["parent"], d["children"], d["level"], d["flags"], d["p"], d["meta"],
                                   d["root"]))
    (desc_r, depth_r, mask_r, data_r), (desc_a, depth_a, mask_a, data_a) = trees
    assert desc_r == desc_a and depth_r == depth_a and mask_r == mask_a
    for nm in data_r:
        wr = [v is not None for v in data_r[nm]]
        assert wr == [v is not None for v in data_a[nm]], nm
        a = np.array([v for v in data_a[nm] if v is not None])
        b = np.array([v for v in data_r[nm] if v is not None])
        if nm == "acti_level":
            assert np.array_equal(a, b)
        elif nm.startswith("p_"):
            assert np.abs(a - b).sum() <= 1e-10 * max(np.abs(b).sum(), 1e-300), nm
        elif nm == "error":
            assert np.all(np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-6 * np.abs(b).max()), nm
        else:
            assert np.all(np.abs(a - b) <= 1e-12 * np.abs(b)), nm


@pytest.mark.gpu
@pytest.mark.parametrize("name,steps", [("euler2", 4), ("ns2", 3), ("multi2", 3), ("multi2_tension_run", 2)])
def test_reference_default_driver_runs_the_adapter(name, steps, tmp_path):
    """DACTI's default_driver (driver/default_driver.hpp), compiled unchanged, keeps and steps its own
    copy of the Integrator: once the reference's, once the GPU adapter. Frames, times, cell counts and
    the observables CSV (with DropEnergy for the multiphase cases) agree."""
    import csv

    if not os.path.exists(CHECK):
        pytest.fail("oracle/_ref/dacti_adapter_check is not built (make -C oracle after building the library)")
    r = subprocess.run([CHECK, os.path.join(GOLDEN, f"{name}.case"), str(tmp_path), str(steps), "--driver-check"],
                       capture_output=True, text=True, timeout=600, env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    rec = [json.loads(x[len("DRIVER "):]) for x in r.stdout.splitlines() if x.startswith("DRIVER ")]
    assert len(rec) == 1
    fr, fg = rec[0]["frames_ref"], rec[0]["frames_gpu"]
    assert len(fr) == steps + 1 and fr == fg  # frame times, indices and cell counts, exactly
    rows_r = list(csv.reader(open(rec[0]["csv_ref"])))
    rows_g = list(csv.reader(open(rec[0]["csv_gpu"])))
    assert rows_r[0] == rows_g[0] and len(rows_r) == len(rows_g) == steps + 1
    for a, b in zip(rows_r[1:], rows_g[1:]):
        assert a[:4] == b[:4]  # time, frame, step, n_cells
        for x, y in zip(a[4:], b[4:]):
            assert abs(float(x) - float(y)) <= 1e-8 * max(abs(float(x)), 1e-300), (a, b)
    if name.startswith("multi"):
        assert rows_r[0][4:] == ["ke", "Etot"]
