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
into the same binary, runs on both integrators after the last step.
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
                        "--adapter-check"], capture_output=True, text=True, timeout=600,
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
