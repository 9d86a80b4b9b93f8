"""Edge cases of the plain form through the C ABI: an empty system, one site
in a box smaller than the cut-off (every neighbour is one of its own images),
dilute sites of which most have no neighbour (ragged, mostly empty lists), and
a compressed lattice whose neighbour count overflows the initial list capacity
(the list grows and is rebuilt).  Results against the oracle as in
tests/test_gpu_parity.py."""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx
from tests.test_gpu_parity import check_state, rel, TOL

pytestmark = pytest.mark.gpu


def _mb():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mapp_b200

    return mapp_b200


def check_forces(s, o, dmd):
    """As tests/test_gpu_parity.check_forces, with the force and virial scales
    floored at 1 (one site among its own images feels no net force: both sides
    give round-off of order 1e-16)."""
    f, en = s.force_calc(1)
    fo, eno = o.force(1)
    assert np.max(np.abs(f - fo)) <= TOL * max(np.max(np.abs(fo)), 1.0)
    assert abs(en[0] - eno[0]) <= TOL * abs(eno[0])
    assert np.max(np.abs(en[1:] - eno[1:])) <= TOL * max(np.max(np.abs(eno[1:])), 1.0)
    assert abs(s.energy_calc() - o.energy()) <= TOL * abs(o.energy())


def _config(kind, s, L, seed=0):
    rng = np.random.default_rng(seed)
    N = len(s)
    if kind == "dmd":
        w = rng.uniform(0.08, 0.15, size=(N, 2))
        c = np.zeros((N, 2))
        c[:, 0] = rng.beta(2, 2, N)
        c[:, 1] = 1 - c[:, 0]
        return fx.Config(L, s, ["A", "B"], [fx.SPECIES_A.mass, fx.SPECIES_B.mass], alpha=1.0 / w**2, c=c)
    return fx.Config(L, s, ["A"], [fx.SPECIES_A.mass], type=np.zeros(N, dtype=np.int32))


def _workload(tmp_path, kind, cfg):
    if kind == "dmd":
        return fx.write_workload(str(tmp_path / "w"), "dmd", cfg=cfg, style="DMD_I")
    # EAM: write the configuration over a generated workload of the same kind
    w = fx.write_workload(str(tmp_path / "w"), "eam", n=2)
    fx.write_cfg(w["cfg_path"], cfg)
    w["cfg"] = cfg
    return w


@pytest.mark.parametrize("kind", ["eam", "dmd"])
def test_empty_system(tmp_path, kind):
    mb = _mb()
    w = fx.write_workload(str(tmp_path / "w"), kind, n=2, **({"style": "DMD_I"} if kind == "dmd" else {}))
    cfg = w["cfg"]
    s = mb.System(w["style"])
    s.set_types(cfg.names, cfg.masses)
    s.set_box(cfg.H())
    s.set_skin(0.5)
    xd = 3 + len(cfg.names) if kind == "dmd" else 3
    if kind == "dmd":
        s.set_atoms(np.zeros((0, xd)), c=np.zeros((0, len(cfg.names))))
    else:
        s.set_atoms(np.zeros((0, 3)), type=np.zeros(0, dtype=np.int32))
    s.coef(w["coef"])
    s.init()
    f, en = s.force_calc(1)
    assert f.shape == (0, xd) and np.all(en == 0.0)
    assert s.energy_calc() == 0.0
    assert s.counts()["npairs"] == 0 and s.counts()["nph"] == 0
    if kind == "dmd":
        s.create_2nd_neigh_lst()
        assert s.c_d_calc().shape == (0, 2)
        cost, g = s.calc_g(np.zeros((0, 2)), 1e-3)
        assert cost == 0.0
    assert s.update_x(np.zeros((0, xd))) == 0


@pytest.mark.parametrize("kind", ["eam", "dmd"])
def test_one_site_in_a_box_smaller_than_the_cut(tmp_path, kind):
    mb = _mb()
    from oracle.restated import Oracle

    cfg = _config(kind, np.array([[0.3, 0.6, 0.1]]), 2.9)
    w = _workload(tmp_path, kind, cfg)
    s = mb.system_from_workload(w)
    o = Oracle(w)
    assert s.counts()["nph"] > 50  # images of the one site fill the cut-off sphere
    check_state(s, o)
    check_forces(s, o, kind == "dmd")


@pytest.mark.parametrize("kind", ["eam", "dmd"])
def test_dilute_sites_mostly_without_neighbours(tmp_path, kind):
    mb = _mb()
    from oracle.restated import Oracle

    rng = np.random.default_rng(4)
    cfg = _config(kind, rng.uniform(0, 1, (60, 3)), 40.0, seed=1)
    w = _workload(tmp_path, kind, cfg)
    s = mb.system_from_workload(w)
    o = Oracle(w)
    sizes, _ = s.neighbor_list()
    assert np.count_nonzero(sizes == 0) > 30
    check_state(s, o)
    check_forces(s, o, kind == "dmd")
    if kind == "dmd":
        # (no c_d comparison: at zero density the embedding slope, and with it
        # the chemical potential and the exp() of the rates, is near overflow)
        s.create_2nd_neigh_lst()
        assert np.array_equal(s.crd(), o.crd())


@pytest.mark.parametrize("kind", ["eam", "dmd"])
def test_compressed_lattice_grows_the_list(tmp_path, kind):
    """About 100-200 half-list neighbours per site: more than the list's
    first capacity (64 EAM / 96 DMD slots), so the device reports the
    overflow and the host regrows and rebuilds."""
    mb = _mb()
    from oracle.restated import Oracle

    a = 2.7
    n = 4
    rng = np.random.default_rng(2)
    x = fx.fcc_sites(n, a) + rng.normal(0, 0.02, (4 * n**3, 3))
    cfg = _config(kind, fx._wrap(x / (n * a)), n * a, seed=3)
    w = _workload(tmp_path, kind, cfg)
    s = mb.system_from_workload(w)
    o = Oracle(w)
    sizes, _ = s.neighbor_list()
    assert sizes.max() > (96 if kind == "dmd" else 64)
    check_state(s, o)
    check_forces(s, o, kind == "dmd")


@pytest.mark.parametrize("kind,kw", [("eam", dict(n=3, sigma=0.05, nt=2, fmt="FS")),
                                     ("dmd", dict(n=3, sigma=0.02, style="DMD_I"))], ids=["eam2", "dmd"])
def test_write_cfg_of_a_system_matches_reference(tmp_path, kind, kw):
    """mg_cfg_write of an initialised system: the same bytes as the reference's
    WriteCFG after its own set-up (the positions after set-up are bit-exact)."""
    mb = _mb()
    from oracle import reference

    if not reference.available():
        pytest.skip("reference harness not built")
    w = fx.write_workload(str(tmp_path / "w"), kind, **kw)
    ref_prefix = str(tmp_path / "ref_out")
    reference.RefRun(w, workdir=str(tmp_path / "ref")).writecfg(ref_prefix, 3).run()
    s = mb.system_from_workload(w)
    path = s.write_cfg(str(tmp_path / "ours"), 3)
    with open(path, "rb") as a, open(ref_prefix + ".00000003.cfg", "rb") as b:
        assert a.read() == b.read()
