"""A batch of independent trees split across ranks, one GPU each.

Each tree is one Integrator of the reference, and trees share nothing. A batch therefore shards with
no exchange at all: every rank builds and steps only its own trees (dg_step_many), and only timings and
counts are combined.

The split needs no communication. Every rank computes the same partition with the
longest-processing-time rule:
- trees are taken in order of decreasing estimated work (ties by index);
- each goes to the rank with the least work so far (ties: lowest rank).
No rank ends more than one tree's work above the mean.

The work estimate of a tree is its active leaves times 2^(max_level - min_level). A global step runs
up to that many substeps of the finest ACTI level, so this bounds the cell updates of a step that
refines everywhere. It is a ranking heuristic: the split only has to be balanced, not exact.
"""
from __future__ import annotations

from typing import List, Sequence


def tree_work(case) -> float:
    """Estimated work of one global step of `case` (a casefile.Case)."""
    leaves = int(case.tree.leaf_mask(active_only=True).sum())
    levels = max(int(case.params.max_level) - int(case.params.min_level), 0)
    return float(leaves) * float(1 << levels)


def partition(work: Sequence[float], world: int) -> List[List[int]]:
    """Tree indices per rank (each list in increasing index order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(work[i])
    return [sorted(p) for p in parts]


def my_trees(work: Sequence[float], rank: int, world: int) -> List[int]:
    """The trees rank `rank` of `world` steps."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return partition(work, world)[rank]
