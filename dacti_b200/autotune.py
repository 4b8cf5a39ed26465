"""Autotuner of the batched step's launch shapes.

A merged batch substep launches each stage kind once for all trees of the running level, over a block
budget (blocks per SM) that the launch splits among the trees in proportion to their work
(csrc/batch.cuh). Too few blocks leave SMs idle on small levels; too many add block scheduling and
tail cost on the many short launches of the fine levels. The best budget differs per stage: the
face-sum and slope stages are long-running and latency bound, the regrid stages are short.

`tune` measures it: on a warmed-up batch it steps once per candidate budget with every stage on that
candidate and per-stage CUDA-event timing, and keeps, per stage kind, the candidate with the least
device time per work item (items: cells, or cell-face lanes). Per-item time makes the global steps,
whose work differs, comparable. The result goes to `launch_table.json` beside this file, keyed by
model and dimension, which `solver.Batch` applies when it is created.
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional, Sequence

TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "launch_table.json")
CANDIDATES = (2, 4, 8, 16, 32)


def key(shape) -> str:
    return f"{shape.model.name.lower()}{shape.dims}"


def table_entry(shape) -> Optional[list]:
    """The tuned blocks-per-SM list of a model and dimension, or None."""
    try:
        with open(TABLE) as f:
            entry = json.load(f).get(key(shape))
    except (OSError, ValueError):
        return None
    return entry["blocks_per_sm"] if entry else None


def tune(cases: Sequence, candidates: Sequence[int] = CANDIDATES, warmup: int = 2, form: str = "mixed",
         rounds: int = 1) -> Dict:
    """Per-stage best launch budget for a batch of `cases` (casefile.Case of one model). Returns
    {"blocks_per_sm": [...], "ns_per_item": {stage: {candidate: ns}}, ...}."""
    from .solver import BATCH_STAGES, Batch, Solver
    solvers = [Solver(c) for c in cases]
    for s in solvers:
        s.set_form(form)
    b = Batch(solvers, launch=[16] * len(BATCH_STAGES))
    for _ in range(warmup):
        b.step()
    b.set_profiling(True)
    b.stage_times()
    per = {st: {} for st in BATCH_STAGES}
    for _ in range(rounds):
        for c in candidates:
            b.set_launch([c] * len(BATCH_STAGES))
            b.step()
            for st, (ms, items) in b.stage_times().items():
                if items > 0:
                    ns = 1e6 * ms / items
                    per[st][c] = min(per[st].get(c, float("inf")), ns)
    b.close()
    for s in solvers:
        s.close()
    best = [min(per[st], key=per[st].get) if per[st] else 16 for st in BATCH_STAGES]
    return {"blocks_per_sm": best, "ns_per_item": {st: {str(k): v for k, v in per[st].items()} for st in per},
            "candidates": list(candidates), "form": form}


def save(shape, result: Dict, workload: str) -> None:
    """Stores a tuning result for a model and dimension in launch_table.json."""
    from .solver import BATCH_STAGES
    try:
        with open(TABLE) as f:
            table = json.load(f)
    except (OSError, ValueError):
        table = {}
    table[key(shape)] = dict(result, workload=workload, stages=list(BATCH_STAGES))
    with open(TABLE, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    from . import cases as _cases
    batch = _cases.riemann_batch(64, seed=3)
    res = tune(batch)
    save(batch[0].shape, res, "64 trees of cases.riemann_batch(seed=3), mixed form")
    print(json.dumps(res["blocks_per_sm"]))
