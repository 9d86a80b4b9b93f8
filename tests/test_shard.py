"""The batched form's split across ranks (mapp_b200.shard): the assignment
of cells to ranks and the gather of per-cell results on rank 0, with two
gloo ranks on the CPU (no GPU)."""
import os
import socket

import numpy as np
import pytest

from mapp_b200 import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_assignment_covers_every_cell_once_and_balances():
    rng = np.random.default_rng(2024)
    costs = np.exp(rng.uniform(np.log(500), np.log(8000), 512)).round()
    for nranks in (1, 2, 3, 4, 8):
        parts = shard.assign_cells(costs, nranks)
        assert len(parts) == nranks
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        assert all(p == sorted(p) for p in parts)
        loads = [costs[p].sum() for p in parts]
        # the longest-processing-time rule leaves at most one largest cell of imbalance
        assert max(loads) - min(loads) <= costs.max()
        assert max(loads) <= costs.sum() / nranks + costs.max()


def test_assignment_is_the_largest_first_rule():
    costs = [5, 9, 2, 9, 7, 1]
    # largest first: cell 1 (9) -> r0, cell 3 (9) -> r1, cell 4 (7) -> r0 (tie 9/9, lower rank),
    # cell 0 (5) -> r1 (16/9), cell 2 (2) -> r1 (16/14), cell 5 (1) -> r0 (tie 16/16)
    assert shard.assign_cells(costs, 2) == [[1, 4, 5], [0, 2, 3]]
    assert shard.assign_cells(costs, 1) == [list(range(6))]
    assert shard.assign_cells([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.assign_cells(costs, 0)


def test_assignment_with_more_ranks_than_cells():
    costs = [3, 1, 2]
    parts = shard.assign_cells(costs, 5)
    # one cell per rank, largest first to the lowest empty rank; the rest idle
    assert parts == [[0], [2], [1], [], []]


def test_job_time_and_rate_on_one_rank():
    """bench.job_rate / job_max: without a process group the job is this rank."""
    import bench

    assert bench.job_max(2.5) == 2.5
    assert bench.job_rate(1000, 10, 2.0, 1) == 1000 * 10 / 2.0


def test_gather_without_process_group_is_local():
    out = shard.gather_results([(1, "b"), (0, "a")], 2)
    assert out == ["a", "b"]
    with pytest.raises(RuntimeError):
        shard.gather_results([(0, "a")], 2)


def _rank_main(rank, world, port, out_dir, costs):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard.assign_cells(costs, world)[rank]
    # a stand-in for one rank's relaxation: per cell its index, rank and "time"
    local = [(k, {"cell": k, "rank": rank, "t_ms": float(costs[k])}) for k in mine]
    t_rank = float(sum(costs[k] for k in mine))
    t_job = bench.job_max(t_rank)
    out = shard.gather_results(local, len(costs))
    if rank == 0:
        with open(os.path.join(out_dir, "gathered.txt"), "w") as fp:
            for r in out:
                fp.write(f"{r['cell']} {r['rank']} {r['t_ms']}\n")
            fp.write(f"job {t_job}\n")
    else:
        assert out is None
    dist.barrier()
    dist.destroy_process_group()


def test_gather_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    costs = [float(c) for c in (800, 4000, 500, 7900, 1200, 3300, 650, 2100, 5000)]
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), costs), nprocs=world,
                       start_method="spawn")
    lines = (tmp_path / "gathered.txt").read_text().split("\n")
    rows = [l.split() for l in lines if l and not l.startswith("job")]
    parts = shard.assign_cells(costs, world)
    assert [int(r[0]) for r in rows] == list(range(len(costs)))
    for r in rows:
        k, rk = int(r[0]), int(r[1])
        assert k in parts[rk]
        assert float(r[2]) == costs[k]
    job = float([l for l in lines if l.startswith("job")][0].split()[1])
    assert job == max(sum(costs[k] for k in p) for p in parts)


def test_gather_rejects_duplicate_and_missing_cells():
    with pytest.raises(RuntimeError, match="two ranks"):
        shard.gather_results([(0, "a"), (1, "b"), (0, "c")], 2)
    with pytest.raises(RuntimeError, match="no rank"):
        shard.gather_results([(0, "a")], 3)
