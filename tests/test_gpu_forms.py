"""Precision form (MG_FORM_FP32) against the FP64 oracle.

Accuracy gates of the precision form: max|dF| <= 1e-4 eV/A over all force
components (positions and alphas), |dE|/site <= 1e-6 eV for the total free
energy.  c_d_calc after a precision-form force call reads FP32 per-pair
densities and pair energies: the chemical potentials are checked at
|d mu| <= 2e-6 eV, and the rates at 2e-5 relative to max|c_d|, because a rate
is an exponential of beta * mu (beta = 1 / kT = 19.3 / eV at 600 K), so the
FP32 rounding of mu (a few 1e-7 eV over about 40 pair terms) moves it by
about 1e-5 relative."""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx

pytestmark = pytest.mark.gpu


def _mb():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mapp_b200

    return mapp_b200


@pytest.mark.parametrize("style,n,nt", [("DMD_I", 6, 2), ("DMD_II", 5, 2), ("DMD", 5, 2), ("DMD_I", 5, 1), ("DMD_I", 10, 2)])
def test_fp32_form_accuracy(tmp_path, style, n, nt):
    mb = _mb()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=n, sigma=0.03, style=style, nt=nt)
    s = mb.system_from_workload(w)
    s.set_form(mb.MG_FORM_FP32)
    o = Oracle(w)
    f, en = s.force_calc(1)
    fo, eno = o.force(1)
    N = w["cfg"].natms
    assert np.max(np.abs(f - fo)) <= 1e-4
    assert abs(en[0] - eno[0]) / N <= 1e-6
    s.create_2nd_neigh_lst()
    o.crd()
    cd, cdo = s.c_d_calc(), o.c_d()
    # n is beta * mu for DMD_I and DMD, mu itself for DMD_II
    to_ev = 1.0 if style == "DMD_II" else 8.617333e-5 * 600.0
    n_gpu = s.vector("n")[:N * nt].reshape(N, nt)
    n_orc = o.vec(2)[:N * nt].reshape(N, nt)
    assert np.max(np.abs(n_gpu - n_orc)) * to_ev <= 2e-6
    assert np.max(np.abs(cd - cdo)) <= 2e-5 * np.max(np.abs(cdo))


def test_fp32_form_rejected_for_eam(tmp_path):
    mb = _mb()
    w = fx.write_workload(str(tmp_path / "w"), "eam", n=3)
    s = mb.system_from_workload(w)
    with pytest.raises(mb.MGError) as e:
        s.set_form(mb.MG_FORM_FP32)
    assert e.value.code == 7


def test_fp32_form_gates_at_256000_sites(tmp_path):
    """The precision form's gates at the size of its workload definition: FCC
    40^3 = 256000 sites of the binary DMD_I system, against the FP64 oracle:
    max|dF| <= 1e-4 eV/A, |dE|/site <= 1e-6 eV, |d mu| <= 2e-6 eV."""
    mb = _mb()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=40, a=3.58, sigma=0.0, style="DMD_I", seed=4321)
    s = mb.system_from_workload(w)
    s.set_form(mb.MG_FORM_FP32)
    o = Oracle(w)
    f, en = s.force_calc(1)
    fo, eno = o.force(1)
    N = w["cfg"].natms
    assert N == 256000
    assert np.max(np.abs(f - fo)) <= 1e-4
    assert abs(en[0] - eno[0]) / N <= 1e-6
    s.create_2nd_neigh_lst()
    o.crd()
    s.c_d_calc()
    o.c_d()
    to_ev = 8.617333e-5 * 600.0
    n_gpu = s.vector("n")[:N * 2]
    n_orc = o.vec(2)[:N * 2]
    assert np.max(np.abs(n_gpu - n_orc)) * to_ev <= 2e-6
