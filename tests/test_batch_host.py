"""Splitting a batch of independent trees across ranks (dacti_b200/batch.py): every tree on exactly one
rank, the split deterministic and balanced to within one tree's work. No GPU needed."""
import numpy as np
import pytest

from dacti_b200 import cases
from dacti_b200.batch import my_trees, partition, tree_work


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_every_tree_once_and_balances(world):
    rng = np.random.default_rng(7)
    work = list(rng.lognormal(3.0, 1.5, 257))
    parts = partition(work, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(work)))
    loads = [sum(work[i] for i in p) for p in parts]
    # longest-processing-time: no rank ends more than one tree's work above the mean
    assert max(loads) - sum(loads) / world <= max(work) + 1e-9
    assert parts == partition(work, world)          # every rank computes the same split
    for r in range(world):
        assert my_trees(work, r, world) == parts[r]


def test_more_ranks_than_trees_and_bad_arguments():
    parts = partition([5.0, 1.0, 3.0], 5)
    assert parts == [[0], [2], [1], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)
    with pytest.raises(ValueError):
        my_trees([1.0], 2, 2)


def test_tree_work_of_the_riemann_batch():
    batch = cases.riemann_batch(6, seed=3)
    w = [tree_work(c) for c in batch]
    for c, x in zip(batch, w):
        leaves = int(c.tree.leaf_mask(active_only=True).sum())
        assert x == leaves * 2 ** (c.params.max_level - c.params.min_level) > 0
    two = partition(w, 2)
    assert sorted(two[0] + two[1]) == list(range(6))
