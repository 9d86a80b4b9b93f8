"""The batched form across GPUs: independent cells split over ranks.

The reference relaxes one system per process (one Min_LBFGS::run per MPI job,
min_l-bfgs.cpp:302, over that job's spatial decomposition).  Cells of the
batched form are independent, so the multi-GPU form is a split of the cells:
each rank (one process per GPU) relaxes its own share with its own Batch in
one graph launch, with no collective on the data path; only the per-cell
results are gathered on rank 0 at the end, and the job's time is the slowest
rank's device time.

Cells are assigned by cost, largest first, each to the rank with the least
load so far (the longest-processing-time rule), so uneven cell sizes do not
leave one GPU with most of the work.  A cell's cost is its site count: at the
workload's fixed density its pair count, and so its force-pass work, is
proportional to it.
"""
from __future__ import annotations

from typing import Iterable, List, Optional, Sequence


def assign_cells(costs: Sequence[float], nranks: int) -> List[List[int]]:
    """Cell indices per rank: cells in decreasing cost (ties: lower index
    first), each to the rank with the least load so far (ties: lower rank).
    Every cell appears once; each rank's list is in increasing cell order."""
    if nranks < 1:
        raise ValueError("nranks must be at least 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * nranks
    out: List[List[int]] = [[] for _ in range(nranks)]
    for k in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        out[r].append(k)
        load[r] += float(costs[k])
    for lst in out:
        lst.sort()
    return out


def cell_costs(cells: Iterable) -> List[float]:
    """Cost of each cell (fixtures.Config): its number of sites."""
    return [float(c.natms) for c in cells]


def gather_results(local: Sequence[tuple], ncells: int, group=None) -> Optional[list]:
    """Gathers (cell index, result) pairs of every rank on rank 0 and returns
    the results in cell order there (None on the other ranks).  Every rank
    must call it.  Without an initialised process group the local pairs are
    the whole job."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        parts = [list(local)]
        rank = 0
    else:
        rank = dist.get_rank(group)
        parts = [None] * dist.get_world_size(group) if rank == 0 else None
        dist.gather_object(list(local), parts, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * ncells
    for part in parts:
        for k, res in part:
            if out[k] is not None:
                raise RuntimeError(f"cell {k} came back from two ranks")
            out[k] = res
    missing = [k for k, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"cells {missing[:8]} came back from no rank")
    return out


def relax_sharded(builder, cells: Sequence, rank: int, world: int, params=(5, 10000, 1e-5, 1e-8, 60),
                  form=None, tuning_cache: Optional[str] = None, warm: bool = False):
    """Relaxes this rank's share of `cells` with one Batch on this rank's GPU
    (with warm, a first relaxation -- launch tuning, first-call set-up -- is
    run and the second one reported).

    Returns (local_stats, local_results): the Batch's relaxation statistics and
    [(cell index, result dict)] for the cells this rank owns.  Gather the
    results with gather_results."""
    from . import Batch

    mine = assign_cells(cell_costs(cells), world)[rank]
    if not mine:
        return {"relax_ms": 0.0, "build_ms": 0.0, "cells": 0, "sites": 0}, []
    B = Batch(builder)
    try:
        for k in mine:
            B.add_cell(cells[k])
        B.set_params(*params)
        if form is not None:
            B.set_form(form)
        if tuning_cache is not None:
            B.set_tuning(True, tuning_cache)
        if warm:
            B.relax()
        st = B.relax()
        res = [(k, B.cell_result(n)[2]) for n, k in enumerate(mine)]
    finally:
        B.close()
    st = dict(st)
    st["cells"] = len(mine)
    st["sites"] = int(sum(cells[k].natms for k in mine))
    return st, res
