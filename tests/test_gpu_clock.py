"""Device Adams and BDF clocks (mg_clock_adams, mg_clock_bdf) against the
restated Clock_Adams and Clock_BDF, themselves pinned bit for bit to the
reference's clock_adams.cpp and clock_bdf.cpp.

The device computes calc_g and the dot products of the conjugate-gradient
solve with parallel sums, so costs and directions differ from the
reference's serial sums in the last bits; the solve's decisions (Armijo
tests, convergence at cost <= 1e-8) are the same on these runs, so both
make the same number of calc_g calls.  Bars: equal calc_g counts,
concentrations within 1e-9 absolute, step costs within 1e-6 relative
(costs near the 1e-8 convergence threshold carry the rounding of a
cancellation) or 1e-16 absolute.

The BDF clock's step-size and order decisions are thresholds on error
estimates computed from the same parallel sums; on these runs they come out
the same as the oracle's, so the step sizes and orders are compared exactly
in count and order and within 1e-9 relative in size, the calc_g counts
exactly, the concentrations within 1e-9 absolute.
"""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx

pytestmark = pytest.mark.gpu


def _lib_or_skip():
    try:
        import torch

        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
    except ImportError:
        pass
    import mapp_b200

    return mapp_b200


def rate_scale(w):
    from oracle.restated import Oracle

    o = Oracle(w)
    o.force()
    o.crd()
    cd = o.c_d()
    return 1.0 / float(np.sqrt(np.mean(cd * cd)))


def _compare(r, o):
    assert r["n_calc_g"] == o["n_calc_g"]
    assert float(np.max(np.abs(r["c"].ravel() - o["c"].ravel()))) <= 1e-9
    assert np.all(np.abs(r["err"] - o["err"]) <= np.maximum(1e-6 * np.abs(o["err"]), 1e-16))


CASES = [
    ("DMD_I", 1, 12, 1e-3),
    ("DMD_I", 3, 15, 1e-3),
    ("DMD_I", 6, 15, 1e-3),
    ("DMD_II", 3, 12, 1e-3),
    ("DMD", 4, 12, 1e-3),
]


@pytest.mark.parametrize("style,order,steps,k", CASES, ids=[f"{s}-o{o}-n{n}" for s, o, n, k in CASES])
def test_clock_adams_matches_oracle(tmp_path, style, order, steps, k):
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style=style)
    dt = k * rate_scale(w)
    s = mb.system_from_workload(w)
    r = s.clock_adams(order, steps, dt)
    o = Oracle(w).clock_adams(order, steps, dt)
    _compare(r, o)


def test_clock_adams_full_size_32000_sites(tmp_path):
    """FCC 20^3 binary DMD_I (32000 sites), order 2, 3 steps of 1e-3 tau."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=20, a=3.58, sigma=0.0, style="DMD_I", seed=4321)
    dt = 1e-3 * rate_scale(w)
    s = mb.system_from_workload(w)
    r = s.clock_adams(2, 3, dt)
    o = Oracle(w).clock_adams(2, 3, dt)
    _compare(r, o)


def test_clock_adams_errors(tmp_path):
    mb = _lib_or_skip()
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=3)
    s = mb.system_from_workload(w)
    with pytest.raises(mb.MGError, match="cannot operate with order"):
        s.clock_adams(7, 2, 1e-6)
    with pytest.raises(mb.MGError):
        s.clock_adams(2, 2, -1.0)
    we = fx.write_workload(str(tmp_path / "e"), "eam", n=3)
    se = mb.system_from_workload(we)
    with pytest.raises(mb.MGError):
        se.clock_adams(2, 2, 1e-6)
    s.set_form(mb.MG_FORM_FP32)
    with pytest.raises(mb.MGError):
        s.clock_adams(2, 2, 1e-6)


def _compare_bdf(r, o):
    assert r["steps"] == o["steps"]
    assert np.array_equal(r["order"], o["order"])
    assert np.all(np.abs(r["del_t"] - o["del_t"]) <= 1e-9 * np.abs(o["del_t"]))
    assert abs(r["t"] - o["t"]) <= 1e-9 * abs(o["t"])
    assert r["n_calc_g"] == o["n_calc_g"]
    assert float(np.max(np.abs(r["c"].ravel() - o["c"].ravel()))) <= 1e-9


BDF_CASES = [
    # style, n, nt, steps, options
    ("DMD_I", 4, 2, 20, {}),
    ("DMD_I", 4, 2, 12, dict(max_order=2, max_iter=20)),
    ("DMD_II", 4, 2, 25, {}),
    ("DMD_II", 4, 2, 60, dict(a_tol=1e-5)),
    ("DMD", 4, 2, 25, dict(a_tol=1e-4)),
    ("DMD_II", 3, 3, 15, dict(initial_del_t=1e-3, m_tol=1e-9, max_del_t=50.0)),
]
BDF_IDS = ["dmd-i-default", "dmd-i-o2-it20", "dmd-ii-default", "dmd-ii-atol1e-5-60", "dmd-atol1e-4", "dmd-ii-3sp"]


@pytest.mark.parametrize("style,n,nt,steps,opts", BDF_CASES, ids=BDF_IDS)
def test_clock_bdf_matches_oracle(tmp_path, style, n, nt, steps, opts):
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=n, nt=nt, sigma=0.02, style=style)
    s = mb.system_from_workload(w)
    r = s.clock_bdf(steps, **opts)
    o = Oracle(w).clock_bdf(steps, **opts)
    _compare_bdf(r, o)


def test_clock_bdf_e_tol_stops_early(tmp_path):
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style="DMD_II")
    e_tol = 0.5 / rate_scale(w) * 4.0
    r = mb.system_from_workload(w).clock_bdf(10, e_tol=e_tol)
    o = Oracle(w).clock_bdf(10, e_tol=e_tol)
    assert o["steps"] < 10
    _compare_bdf(r, o)


def test_clock_bdf_full_size_32000_sites(tmp_path):
    """FCC 20^3 binary DMD_II (32000 sites), 20 steps from the default first
    step: the order rises to 2 on the way."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=20, a=3.58, sigma=0.0, style="DMD_II", seed=4321)
    r = mb.system_from_workload(w).clock_bdf(20)
    o = Oracle(w).clock_bdf(20)
    _compare_bdf(r, o)
    assert o["order"].max() == 2


def test_clock_bdf_errors(tmp_path):
    mb = _lib_or_skip()
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=3, sigma=0.02)
    s = mb.system_from_workload(w)
    with pytest.raises(mb.MGError, match="max_order should be larger than zero"):
        s.clock_bdf(2, max_order=0)
    with pytest.raises(mb.MGError, match="no of steps"):
        s.clock_bdf(0)
    with pytest.raises(mb.MGError, match="max_del_t should be larger than min_del_t"):
        s.clock_bdf(2, min_del_t=1.0, max_del_t=0.5)
    with pytest.raises(mb.MGError, match="initial_del_t should be larger than zero"):
        s.clock_bdf(2, initial_del_t=0.0)
    with pytest.raises(mb.MGError, match="max_order above 12"):
        s.clock_bdf(2, max_order=13)
    tau = rate_scale(w)
    with pytest.raises(mb.MGError, match="min_del_t"):
        s.clock_bdf(5, max_order=2, a_tol=1e-30, initial_del_t=1e-2 * tau, min_del_t=1e-2 * tau,
                    max_del_t=2e-2 * tau)
    we = fx.write_workload(str(tmp_path / "e"), "eam", n=3)
    with pytest.raises(mb.MGError):
        mb.system_from_workload(we).clock_bdf(2)


def test_clock_bdf_predictor_stall(tmp_path):
    """Where the reference's clamped predictor retry loop would never end (the
    predictor leaves [0, 1] even at min_del_t) the device clock stops with
    MG_ERR_DOMAIN, as the oracle does: here the first step may not be
    shorter than 10 tau, which carries most sites out of the box."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style="DMD_I")
    tau = rate_scale(w)
    opts = dict(max_order=2, initial_del_t=10.0 * tau, min_del_t=10.0 * tau, max_del_t=20.0 * tau)
    with pytest.raises(ValueError, match="even at min_del_t"):
        Oracle(w).clock_bdf(5, **opts)
    with pytest.raises(mb.MGError, match="even at min_del_t"):
        mb.system_from_workload(w).clock_bdf(5, **opts)


@pytest.mark.parametrize("fail", [False, True], ids=["after-return", "after-domain-error"])
def test_lists_after_clock(tmp_path, fail):
    """While a clock runs, c_d_calc and calc_g walk the active-pair sublist of
    the clock's initial force_calc.  After the clock returns -- normally, or
    with MG_ERR_DOMAIN from the predictor stall -- they walk the full list
    again: the sites are then moved and the concentrations reset, and
    c_d_calc and calc_g must match the oracle on the new state at 1e-10."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style="DMD_I")
    s = mb.system_from_workload(w)
    if fail:
        tau = rate_scale(w)
        with pytest.raises(mb.MGError, match="even at min_del_t"):
            s.clock_bdf(5, max_order=2, initial_del_t=10.0 * tau, min_del_t=10.0 * tau, max_del_t=20.0 * tau)
    else:
        s.clock_bdf(5)
    o = Oracle(w)
    o.force(1)
    N = w["cfg"].natms
    x1 = s.get_x()
    x1[:, :3] += np.random.default_rng(9).normal(0, 0.08, (N, 3))
    c = w["cfg"].c.copy()
    assert s.update_x(x1) == o.update_x(x1)
    s.update_c(c)
    o.update_c(c)
    s.force_calc(1)
    o.force(1)
    s.create_2nd_neigh_lst()
    o.crd()
    cd, cdo = s.c_d_calc(), o.c_d()
    assert float(np.max(np.abs(cd - cdo))) <= 1e-10 * float(np.max(np.abs(cdo)))
    a = np.random.default_rng(3).normal(0, 1e-3, (N, w["cfg"].c.shape[1]))
    cost, g = s.calc_g(a, 0.01)
    cost_o, g_o = o.calc_g(a, 0.01)
    assert abs(cost - cost_o) <= 1e-10 * abs(cost_o)
    assert float(np.max(np.abs(g - g_o))) <= 1e-10 * float(np.max(np.abs(g_o)))
