"""Pins the BDF clock restatement (orc_clock_bdf in oracle/mapp_oracle.c) to
the reference's own Clock_BDF (clock_bdf.cpp) run by the compiled harness:
the concentrations after the run and the final time agree bit for bit and
both make the same number of calc_g calls, for the three DMD styles, one and
two species, default and non-default options, runs where the order rises and
falls, and a run that the e_tol test ends early.

Clock_BDF::solve reads a local time it never sets (clock_bdf.cpp:838-854);
the reference built with gcc -O2 evaluates it as 0.0, and the restatement
does the same -- these pins are what shows that reading."""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx
from oracle import reference
from oracle.restated import Oracle

pytestmark = pytest.mark.skipif(not reference.available(), reason="reference harness not built")


def rms_c_d(w):
    o = Oracle(w)
    o.force()
    o.crd()
    cd = o.c_d()
    return float(np.sqrt(np.mean(cd * cd)))


CASES = [
    # style, n, nt, steps, options
    ("DMD_I", 4, 2, 20, {}),
    ("DMD_I", 4, 2, 12, dict(max_order=2, max_iter=20)),
    ("DMD_II", 4, 2, 25, {}),                   # the order rises to 2 and falls back
    ("DMD_II", 4, 2, 60, dict(a_tol=1e-5)),
    ("DMD", 4, 2, 25, dict(a_tol=1e-4)),
    ("DMD_I", 3, 3, 6, dict(slope=0.3, gamma_red=0.7, min_gamma=1e-8)),
    ("DMD_II", 3, 3, 15, dict(initial_del_t=1e-3, m_tol=1e-9, max_del_t=50.0)),
]
IDS = ["dmd-i-default", "dmd-i-o2-it20", "dmd-ii-default", "dmd-ii-atol1e-5-60", "dmd-atol1e-4", "dmd-i-3sp-ls",
       "dmd-ii-3sp-dt0"]


@pytest.mark.parametrize("style,n,nt,steps,opts", CASES, ids=IDS)
def test_clock_bdf_bit_exact(tmp_path, style, n, nt, steps, opts):
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=n, nt=nt, sigma=0.02, style=style)
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.bdf(steps, **opts)
    r = ref.run()["bdf"]
    res = Oracle(w).clock_bdf(steps, **opts)
    assert np.array_equal(res["c"].ravel(), r["c"]), f"max |dc| = {np.max(np.abs(res['c'].ravel() - r['c']))}"
    assert res["n_calc_g"] == r["meta"]["n_calc_g"]
    assert res["t"] == float(r["meta"]["t"])
    assert res["steps"] == steps
    assert np.all((res["c"] >= 0.0) & (res["c"] <= 1.0))
    assert np.all(np.diff(np.r_[0.0, res["order"]]) <= 1)


def test_clock_bdf_order_changes(tmp_path):
    """The DMD_II default run above changes order: the history records it."""
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style="DMD_II")
    res = Oracle(w).clock_bdf(25)
    assert res["order"].max() == 2 and res["order"][-1] == 1
    assert abs(np.sum(res["del_t"]) - res["t"]) <= 1e-12 * res["t"]


def test_clock_bdf_e_tol_stops_early(tmp_path):
    """rms(c_d) / e_tol < 1 ends the run (clock_bdf.cpp:502, 866-868)."""
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style="DMD_II")
    e_tol = 2.0 * rms_c_d(w)
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.bdf(10, e_tol=e_tol)
    r = ref.run()["bdf"]
    res = Oracle(w).clock_bdf(10, e_tol=e_tol)
    assert res["steps"] < 10
    assert np.array_equal(res["c"].ravel(), r["c"])
    assert res["n_calc_g"] == r["meta"]["n_calc_g"]
    assert res["t"] == float(r["meta"]["t"])


@pytest.mark.parametrize("opts,msg", [
    (dict(max_order=0), "max_order should be larger than zero"),
    (dict(gamma_red=1.0), "gamma_red should be between zero and one"),
    (dict(min_del_t=1.0, max_del_t=0.5), "max_del_t should be larger than min_del_t"),
    (dict(initial_del_t=-1.0), "initial_del_t should be larger than zero"),
])
def test_clock_bdf_bad_options(tmp_path, opts, msg):
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=3)
    ref = reference.RefRun(w, str(tmp_path / "ref"), init=False)
    ref.bdf(2, **opts)
    with pytest.raises(RuntimeError, match=msg):
        ref.run()
    with pytest.raises(ValueError, match=msg):
        Oracle(w).clock_bdf(2, **opts)


def test_clock_bdf_stall_at_min_del_t(tmp_path):
    """A step whose error test fails at min_del_t is retried at the same size
    for ever by the reference (clock_bdf.cpp:513-540); the restatement stops
    with an error instead (the reference is not run: it would not end)."""
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=3, sigma=0.02, style="DMD_I")
    tau = 1.0 / rms_c_d(w)
    with pytest.raises(ValueError, match="min_del_t"):
        Oracle(w).clock_bdf(5, max_order=2, a_tol=1e-30, initial_del_t=1e-2 * tau, min_del_t=1e-2 * tau,
                            max_del_t=2e-2 * tau)


def test_clock_bdf_predictor_stall(tmp_path):
    """DMD_I's calc_g never refreshes c_d (ff_dmd_I.cpp:2402-2674), so
    Clock_BDF keeps predicting with the initial rates (clock_bdf.cpp:565) and
    on this undisplaced lattice drives a site against the [0, 1] box; the
    reference's clamped retry loop (clock_bdf.cpp:504-510) then repeats at
    min_del_t for ever (the compiled reference was seen still running after
    120 s).  The restatement stops with an error at that point."""
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, a=3.58, sigma=0.0, style="DMD_I", seed=4321)
    tau = 1.0 / rms_c_d(w)
    with pytest.raises(ValueError, match="even at min_del_t"):
        Oracle(w).clock_bdf(100, max_order=2, initial_del_t=1e-3 * tau)
