"""The autotuner's table: a result saved for a model and dimension comes back for that model's batches,
and a missing table or entry means the library's default budgets."""
import json

from dacti_b200 import autotune
from dacti_b200.models import ModelId, ModelShape
from dacti_b200.solver import BATCH_STAGES


def test_table_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "TABLE", str(tmp_path / "t.json"))
    e2 = ModelShape(ModelId.EULER, 2)
    m3 = ModelShape(ModelId.MULTI, 3)
    assert autotune.table_entry(e2) is None
    res = {"blocks_per_sm": [4, 8, 16, 8, 4, 8, 2, 2, 4, 2], "ns_per_item": {}, "candidates": [2, 4, 8, 16],
           "form": "mixed"}
    autotune.save(e2, res, "test")
    assert autotune.table_entry(e2) == res["blocks_per_sm"]
    assert autotune.table_entry(m3) is None
    table = json.load(open(tmp_path / "t.json"))
    assert table["euler2"]["stages"] == list(BATCH_STAGES) and table["euler2"]["workload"] == "test"
    assert len(BATCH_STAGES) == 10
