"""Pins the Nose-Hoover NVT restatement (orc_md_nh in oracle/mapp_oracle.c) to
the reference's own MD_NH (md_nh.cpp) run by the compiled harness: positions,
velocities, the final force_calc energy and virial agree bit for bit after
hundreds of steps with several list rebuilds, for create_vel and for given
velocities (init_vel), with default and non-default chain settings."""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx
from oracle import reference
from oracle.restated import Oracle

pytestmark = pytest.mark.skipif(not reference.available(), reason="reference harness not built")

DT = 0.0982269     # 1 fs in the reference's sqrt(amu A^2 / eV) time unit
KB = 8.617333e-5   # eV / K

CASES = [
    # kind, workload kw, T, period, steps, seed (0: given velocities), eta_iteration, eta_chains
    ("eam", dict(n=4, seed=7), 300.0, 0.1, 300, 5, 1, 3),
    ("eam", dict(n=4, nt=2, fmt="FS", seed=8), 600.0, 0.05, 200, 0, 2, 4),
    ("fs", dict(n=4, nt=2, seed=9), 450.0, 0.2, 150, 11, 1, 5),
    ("eam", dict(n=4, seed=7, skin=0.1), 900.0, 1.0, 300, 5, 1, 3),
]


def _same(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    assert a.shape == b.shape
    assert np.array_equal(a, b), f"max |diff| = {np.max(np.abs(a - b))}"


@pytest.mark.parametrize("kind,kw,T,period,steps,seed,it,ch", CASES,
                         ids=["eam-create_vel", "eam2-init_vel-it2-ch4", "fs2-create_vel-ch5", "eam-skin0.1-rebuilds"])
def test_md_nh_bit_exact(tmp_path, kind, kw, T, period, steps, seed, it, ch):
    w = fx.write_workload(str(tmp_path / "w"), kind, **kw)
    n = w["cfg"].natms
    xd = None
    if seed == 0:
        xd = np.random.default_rng(3).normal(0.0, 0.02, size=(n, 3))
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.md(T, period, steps, DT, KB, xd=xd, seed=seed, eta_iteration=it, eta_chains=ch)
    r = ref.run()["md"]
    o = Oracle(w)
    res = o.md_nh(T, period, steps, DT, KB, xd=xd, seed=seed, eta_iteration=it, eta_chains=ch)
    _same(res["x"], r["x"])
    _same(res["xd"], r["xd"])
    _same([res["energy"], *res["virial"]], r["meta"]["en"])
    # the thermostat holds the kinetic temperature near its target
    assert abs(res["t"] - T) < 0.5 * T


def test_md_nh_zero_velocities_rejected(tmp_path):
    """init_vel aborts on all-zero velocities (md_nh.cpp:1331-1334); so does the restatement."""
    w = fx.write_workload(str(tmp_path / "w"), "eam", n=3)
    n = w["cfg"].natms
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.md(300.0, 0.1, 5, DT, KB, xd=np.zeros((n, 3)))
    with pytest.raises(RuntimeError, match="initial velocities are zero"):
        ref.run()
    with pytest.raises(ValueError):
        Oracle(w).md_nh(300.0, 0.1, 5, DT, KB, xd=np.zeros((n, 3)))
