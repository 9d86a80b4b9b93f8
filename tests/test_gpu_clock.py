"""Device Adams clock (mg_clock_adams) against the restated Clock_Adams,
itself pinned bit for bit to the reference's clock_adams.cpp.

The device computes calc_g and the dot products of the conjugate-gradient
solve with parallel sums, so costs and directions differ from the
reference's serial sums in the last bits; the solve's decisions (Armijo
tests, convergence at cost <= 1e-8) are the same on these runs, so both
make the same number of calc_g calls.  Bars: equal calc_g counts,
concentrations within 1e-9 absolute, step costs within 1e-6 relative
(costs near the 1e-8 convergence threshold carry the rounding of a
cancellation) or 1e-16 absolute.
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
