"""The oracle's L-BFGS restatement (orc_lbfgs) pinned to the reference's own
Min_LBFGS run, and the property of the reference's DMD model that bounds
every energy-line-search relaxation of it."""
import tempfile

import numpy as np
import pytest

from mapp_b200 import fixtures as fx
from oracle import reference
from oracle.restated import Oracle

needs_ref = pytest.mark.skipif(not reference.available(), reason="reference harness not built")


@needs_ref
@pytest.mark.parametrize("style", ["DMD_I", "DMD_II", "DMD"])
def test_lbfgs_restatement_matches_reference_bit_for_bit(style):
    """One species: 60 iterations of Min_LBFGS (m = 5), every force_calc
    energy and the final x identical."""
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=3, sigma=0.03, nt=1, style=style)
    r = reference.RefRun(w, init=False).lbfgs(5, 60, 1e-12).run()["lb"]
    o = Oracle(w).lbfgs(5, 60, 1e-12)
    assert o["code"] == int(r["meta"]["code"]) == 4  # MIN_F_MAX_ITER
    assert np.array_equal(o["energies"], r["ehist"])
    assert np.array_equal(o["x"].ravel(), r["x"])


@needs_ref
def test_lbfgs_two_species_reference_fails_its_first_line_search():
    """Two species: the reference's energy_calc sums only same-species phi
    (ff_dmd_I.cpp:508), so the line search compares energies of another
    function than force_calc's; its first line search halves until the step
    underflows (1074 energy_calc calls) and stops with LS_F_ALPHAMIN.  The
    restatement reproduces that exactly."""
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=3, sigma=0.03, style="DMD_I")
    r = reference.RefRun(w, init=False).lbfgs(5, 20, 1e-12).run()["lb"]
    o = Oracle(w).lbfgs(5, 20, 1e-12)
    assert int(r["meta"]["code"]) == o["code"] == 3
    assert int(r["meta"]["n_energy"]) == 1074
    assert np.array_equal(o["energies"], r["ehist"])


def _fd_force(o, x, i, q, eps):
    xp = x.copy()
    xp[i, q] += eps
    o.update_x(xp)
    ep = o.force(1)[1][0]
    xm = x.copy()
    xm[i, q] -= eps
    o.update_x(xm)
    em = o.force(1)[1][0]
    o.update_x(x)
    return -(ep - em) / (2 * eps)


def test_reference_dmd_forces_are_not_the_energy_gradient():
    """Why no relaxation of the reference's DMD model reaches max|F| < 1e-5:
    its forces are not minus the gradient of its own force_calc energy.
    One species: the finite-difference derivative of the energy and the force
    differ by a few % (at n = 3 and n = 10 quadrature nodes alike); the r and
    alpha derivatives are Gaussian identities of the exact smearing integral
    applied to the n-node quadrature.  Two species: pass 2
    pairs the density derivative of slot type2rho[jtype][itype] with
    dE[i][itype] (ff_dmd_I.cpp:376), the value pass 1 computed with the
    transposed species' widths, so the mismatch is of order one."""
    def worst(nt, nq):
        w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=3, sigma=0.03, nt=nt, n_quad=nq, style="DMD_I")
        o = Oracle(w)
        x = o.x_all()[: o.counts()["natms"]].copy()
        f, _ = o.force(1)
        rel = []
        for i in (5, 41, 77):
            for q in (0, 1, 2):
                fd = _fd_force(o, x, i, q, 1e-5)
                rel.append(abs(fd - f[i, q]) / max(abs(fd), 1e-3))
        return max(rel)

    e1_3, e1_10, e2_10 = worst(1, 3), worst(1, 10), worst(2, 10)
    assert 1e-3 < e1_3 < 0.2
    assert 1e-3 < e1_10 < 0.2
    assert e2_10 > 0.2


@needs_ref
@pytest.mark.parametrize("style", ["DMD_I", "DMD_II", "DMD"])
def test_cg_restatement_matches_reference_bit_for_bit(style):
    """One species: 60 iterations of the reference's Min_CG (Polak-Ribiere with
    the same backtracking line search), every force_calc energy and the final
    x identical to orc_cg's."""
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=3, sigma=0.03, nt=1, style=style)
    r = reference.RefRun(w, init=False).cg(60, 1e-12).run()["cg"]
    o = Oracle(w).cg(60, 1e-12)
    assert o["code"] == int(r["meta"]["code"])
    assert np.array_equal(o["energies"], r["ehist"])
    assert np.array_equal(o["x"].ravel(), r["x"])


@needs_ref
def test_cg_two_species_reference_fails_its_first_line_search():
    """Two species: Min_CG's line search meets the same energy_calc defect as
    Min_LBFGS's and stops with LS_F_ALPHAMIN; the restatement agrees."""
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=3, sigma=0.03, style="DMD_I")
    r = reference.RefRun(w, init=False).cg(20, 1e-12).run()["cg"]
    o = Oracle(w).cg(20, 1e-12)
    assert int(r["meta"]["code"]) == o["code"] == 3
    assert np.array_equal(o["energies"], r["ehist"])
