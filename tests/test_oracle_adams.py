"""Pins the Adams clock restatement (orc_clock_adams in oracle/mapp_oracle.c)
to the reference's own Clock_Adams (clock_adams.cpp) run by the compiled
harness: the concentrations after the run agree bit for bit and both make the
same number of calc_g calls, for the three DMD styles and orders 1 to 6.

The time step is set from the system's own rate scale tau = 1 / rms(c_d) at
the initial state: dt = 1e-3 tau is the resolved regime (each step's
conjugate-gradient solve converges in a few calc_g calls), 1e-2 tau the
regime where the solves stall against the box constraints."""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx
from oracle import reference
from oracle.restated import Oracle

pytestmark = pytest.mark.skipif(not reference.available(), reason="reference harness not built")


def rate_scale(w):
    o = Oracle(w)
    o.force()
    o.crd()
    cd = o.c_d()
    return 1.0 / float(np.sqrt(np.mean(cd * cd)))


CASES = [
    # style, order, steps, dt / tau
    ("DMD_I", 1, 12, 1e-3),
    ("DMD_I", 3, 15, 1e-3),
    ("DMD_I", 6, 15, 1e-3),
    ("DMD_I", 2, 10, 1e-2),
    ("DMD_II", 3, 12, 1e-3),
    ("DMD", 4, 12, 1e-3),
]


@pytest.mark.parametrize("style,order,steps,k", CASES, ids=[f"{s}-o{o}-n{n}-{k:g}" for s, o, n, k in CASES])
def test_clock_adams_bit_exact(tmp_path, style, order, steps, k):
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style=style)
    dt = k * rate_scale(w)
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.adams(order, steps, dt)
    r = ref.run()["adams"]
    res = Oracle(w).clock_adams(order, steps, dt)
    assert np.array_equal(res["c"].ravel(), r["c"]), f"max |dc| = {np.max(np.abs(res['c'].ravel() - r['c']))}"
    assert res["n_calc_g"] == r["meta"]["n_calc_g"]
    assert np.all((res["c"] >= 0.0) & (res["c"] <= 1.0))


def test_clock_adams_order_out_of_range(tmp_path):
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=3)
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.adams(7, 2, 1e-6)
    with pytest.raises(RuntimeError, match="cannot operate with order"):
        ref.run()
    with pytest.raises(ValueError):
        Oracle(w).clock_adams(7, 2, 1e-6)
