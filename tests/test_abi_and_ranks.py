"""CPU checks of the boundary and of the multi-rank host logic: the library
loads and exports every entry point the public header declares (nothing is
called), the Python mirror binds them all, and bench.py's whole-job
aggregation is right over two gloo ranks."""
import ctypes
import os
import re
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mapp_b200.h")
LIB = os.path.join(ROOT, "mapp_b200", "libmapp_b200.so")


def declared_entry_points():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mg_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_entry_points()
    for must in ("mg_create", "mg_ff_force_calc", "mg_ff_energy_calc", "mg_ff_c_d_calc", "mg_ff_calc_g",
                 "mg_neighbor_create_list", "mg_atoms_update_x", "mg_batch_relax", "mg_mlp_train",
                 "mg_fs_energy_noalloc"):
        assert must in names


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_library_exports_every_declared_entry_point():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_entry_points() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_bdf_defaults_are_the_references():
    """mg_bdf_defaults (host code, no device call) fills Clock_BDF's
    constructor defaults (clock_bdf.cpp:14-24), the same ones the oracle's
    restatement uses."""
    import mapp_b200 as mb
    from oracle.restated import BDF_DEFAULTS

    o = mb.BdfOpts()
    mb.load_library().mg_bdf_defaults(ctypes.byref(o))
    for k, v in BDF_DEFAULTS.items():
        assert getattr(o, k) == v, k


def test_python_mirror_binds_every_entry_point():
    import mapp_b200

    assert set(declared_entry_points()) <= set(mapp_b200.SIGNATURES)


def declared_arg_counts():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name, args in re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mg_\w+)\s*\(([^)]*)\)\s*;", text, flags=re.M | re.S):
        args = " ".join(args.split())
        out[name] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_python_mirror_argument_counts_match_the_header():
    """Each ctypes signature of the mirror takes as many arguments as the
    header's declaration, so a changed entry point cannot be called with a
    stale argument list."""
    import mapp_b200

    counts = declared_arg_counts()
    assert len(counts) == len(declared_entry_points())
    wrong = {n: (c, len(mapp_b200.SIGNATURES[n][1])) for n, c in counts.items()
             if len(mapp_b200.SIGNATURES[n][1]) != c}
    assert not wrong, wrong


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t_local = 0.5 + rank  # seconds: rank 1 is the slowest
    t = bench.job_max(t_local)
    rate = bench.job_rate(32000, 10, t, world)
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as fp:
        fp.write(f"{t} {rate}\n")
    dist.barrier()
    dist.destroy_process_group()


def test_whole_job_rate_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    vals = [tuple(map(float, (tmp_path / f"r{r}.txt").read_text().split())) for r in range(world)]
    for t, rate in vals:
        assert t == 1.5  # the max over ranks, seen by every rank
        assert rate == pytest.approx(world * 32000 * 10 / 1.5)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(gpus=2, steps=1, warmup=0, impl="reference", cells=3, cpu_reps=1, no_cpu=True)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""
