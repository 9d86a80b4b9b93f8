"""GPU parity: the mapp_b200 CUDA library, called through its C ABI, against the
restated oracle (itself pinned bit for bit to the compiled reference).

Bars (plain FP64 form):
  * ghost images, owned positions after a rebuild and the half neighbour list
    (as a sorted (i, j) set) are bit-exact;
  * forces: max|dF| / max|F| <= 1e-10; energies, virials, chemical-potential
    rates and calc_g gradients: relative (or relative to the max element)
    <= 1e-10.
"""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _lib_or_skip():
    try:
        import torch

        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
    except ImportError:
        pass
    import mapp_b200

    return mapp_b200


def roots(o):
    c = o.counts()
    src = o.ghost_src()
    N = c["natms"]
    r = np.zeros(len(src), dtype=np.int64)
    for k, s in enumerate(src):
        r[k] = s if s < N else r[s - N]
    return r


def pairset(sizes, flat):
    i = np.repeat(np.arange(len(sizes)), sizes)
    return np.unique(np.stack([i, flat]).T, axis=0)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    scale = max(np.max(np.abs(b)), 1e-300)
    return np.max(np.abs(a - b)) / scale


def check_state(s, o):
    c = s.counts()
    oc = o.counts()
    assert (c["natms"], c["nph"], c["npairs"]) == (oc["natms"], oc["nph"], oc["npairs"])
    N = c["natms"]
    xo = o.x_all()
    assert np.array_equal(s.get_x(), xo[:N])
    gx, gown = s.ghosts()
    assert np.array_equal(gx, xo[N:])
    assert np.array_equal(gown, roots(o))
    ns, fl = s.neighbor_list()
    ons, ofl = o.neighbor_list()
    assert np.array_equal(ns, ons)
    assert np.array_equal(pairset(ns, fl), pairset(ons, ofl))


def check_forces(s, o, dmd):
    f, en = s.force_calc(1)
    fo, eno = o.force(1)
    assert rel(f, fo) <= TOL
    assert abs(en[0] - eno[0]) <= TOL * abs(eno[0])
    assert rel(en[1:], eno[1:]) <= TOL
    e = s.energy_calc()
    eo = o.energy()
    assert abs(e - eo) <= TOL * abs(eo)
    return f


CASES = [
    ("eam", dict(n=4)),
    ("eam", dict(n=10)),
    ("eam", dict(n=5, nt=2, fmt="FS")),
    ("eam", dict(n=5, fmt="FuncFL")),
    ("eam", dict(n=4, nt=2, fmt="FuncFL")),
    ("fs", dict(n=4, nt=2)),
    ("fs", dict(n=6)),
    ("dmd", dict(n=4, sigma=0.02, style="DMD_I")),
    ("dmd", dict(n=6, sigma=0.03, style="DMD_I")),
    ("dmd", dict(n=4, sigma=0.02, style="DMD_II")),
    ("dmd", dict(n=4, sigma=0.02, style="DMD")),
    ("dmd", dict(n=3, sigma=0.02, style="DMD_I", nt=1)),
    ("dmd", dict(n=4, sigma=0.02, style="DMD_I", nt=3)),
]


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{k}-{'-'.join(f'{a}{b}' for a, b in v.items())}" for k, v in CASES])
def test_gpu_matches_oracle(tmp_path, kind, kw):
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), kind, **kw)
    s = mb.system_from_workload(w)
    o = Oracle(w)
    N = w["cfg"].natms
    dmd = w["cfg"].dmd
    check_state(s, o)
    check_forces(s, o, dmd)
    if dmd:
        nt = len(w["cfg"].names)
        s.create_2nd_neigh_lst()
        assert np.array_equal(s.crd(), o.crd())
        assert rel(s.c_d_calc(), o.c_d()) <= TOL
        rng = np.random.default_rng(3)
        a = rng.normal(0, 0.01, (N, nt))
        for alpha in (1e-3, 0.05):
            cost, g = s.calc_g(a, alpha)
            cost_o, g_o = o.calc_g(a, alpha)
            assert abs(cost - cost_o) <= TOL * abs(cost_o)
            assert rel(g, g_o) <= TOL
            cost_chk, _ = s.calc_g(a, alpha, chk=1)
            assert abs(cost_chk - cost_o) <= TOL * abs(cost_o)
    # update_0: a move inside the skin refreshes ghosts, a larger one rebuilds
    x0 = s.get_x()
    rng = np.random.default_rng(5)
    x1 = x0.copy()
    x1[:, :3] += rng.normal(0, 0.05, (N, 3))
    assert s.update_x(x1) == o.update_x(x1) == 0
    gx, _ = s.ghosts()
    assert np.array_equal(gx, o.x_all()[N:])
    check_forces(s, o, dmd)
    x2 = x1.copy()
    x2[: max(1, N // 50), :3] += 0.7
    assert s.update_x(x2) == o.update_x(x2) == 1
    check_state(s, o)
    check_forces(s, o, dmd)
    if dmd:
        c = w["cfg"].c.copy()
        c[:, 0] = np.clip(c[:, 0] + rng.normal(0, 0.05, N), 0.01, 0.99)
        if c.shape[1] > 1:
            c[:, 1] = 1.0 - c[:, 0] if c.shape[1] == 2 else c[:, 1]
        s.update_c(c)
        o.update_c(c)
        check_forces(s, o, dmd)
        s.create_2nd_neigh_lst()
        o.crd()
        assert rel(s.c_d_calc(), o.c_d()) <= TOL


@pytest.mark.parametrize("kind,kw", [("eam", dict(n=4)), ("dmd", dict(n=4, sigma=0.02, style="DMD_I"))],
                         ids=["eam", "dmd"])
def test_gpu_update_x_without_waiting(tmp_path, kind, kw):
    """update_x with no rebuilt flag asked for leaves the skin test pending:
    force_calc reads it with its results and, past the skin, rebuilds and
    evaluates again; other entry points settle it first. Forces, lists and
    ghosts match the oracle's update_0 either way."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), kind, **kw)
    s = mb.system_from_workload(w)
    o = Oracle(w)
    N = w["cfg"].natms
    dmd = w["cfg"].dmd
    x0 = s.get_x()
    rng = np.random.default_rng(11)
    x1 = x0.copy()
    x1[:, :3] += rng.normal(0, 0.05, (N, 3))
    assert s.update_x(x1, report=False) is None
    assert o.update_x(x1) == 0
    check_forces(s, o, dmd)
    check_state(s, o)
    # past the skin: force_calc finds out and rebuilds
    x2 = x1.copy()
    x2[: max(1, N // 50), :3] += 0.7
    s.update_x(x2, report=False)
    assert o.update_x(x2) == 1
    check_forces(s, o, dmd)
    check_state(s, o)
    # past the skin again, settled by a list query instead of force_calc
    x3 = x2.copy()
    x3[-max(1, N // 50):, :3] -= 0.7
    s.update_x(x3, report=False)
    assert o.update_x(x3) == 1
    check_state(s, o)
    check_forces(s, o, dmd)
    # two updates in a row: the second settles the first
    s.update_x(x2, report=False)
    s.update_x(x3, report=False)
    assert o.update_x(x2) == 1 and o.update_x(x3) == 1
    check_forces(s, o, dmd)


BOXES = [
    ("eam", dict(n=4, sigma=0.05), 4 * 3.615, (1.3, -0.9, 0.7)),
    ("dmd", dict(n=4, sigma=0.02, style="DMD_I"), 4 * 3.58, (0.8, 0.0, -0.6)),
    ("eam", dict(n=1, sigma=0.05), 3.615, (0.0, 0.0, 0.0)),
    ("dmd", dict(n=1, sigma=0.02, style="DMD_I"), 3.58, (0.0, 0.0, 0.0)),
    ("dmd", dict(n=2, sigma=0.02, style="DMD_II"), 2 * 3.58, (0.4, 0.0, 0.3)),
]


@pytest.mark.parametrize("kind,kw,L,tilt", BOXES,
                         ids=["eam-sheared", "dmd-sheared", "eam-1cell", "dmd-1cell", "dmd-2cell-sheared"])
def test_gpu_matches_oracle_sheared_and_small_boxes(tmp_path, kind, kw, L, tilt):
    """Triclinic boxes and boxes smaller than the cut-off (several ghost passes
    per direction), the cases the oracle is pinned on in
    tests/test_oracle_vs_reference.py."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    H = np.array([[L, 0.0, 0.0], [tilt[0], L, 0.0], [tilt[1], tilt[2], L]])
    w = fx.write_workload(str(tmp_path / "w"), kind, box=H, **kw)
    s = mb.system_from_workload(w)
    o = Oracle(w)
    check_state(s, o)
    check_forces(s, o, w["cfg"].dmd)
    if w["cfg"].dmd:
        s.create_2nd_neigh_lst()
        assert np.array_equal(s.crd(), o.crd())
        assert rel(s.c_d_calc(), o.c_d()) <= TOL
    N = w["cfg"].natms
    x1 = s.get_x()
    x1[:, :3] += np.random.default_rng(9).normal(0, 0.05, (N, 3))
    assert s.update_x(x1) == o.update_x(x1) == 0
    check_forces(s, o, w["cfg"].dmd)


def test_gpu_dmd_full_size_32000(tmp_path):
    """The binary DMD_I system at its benchmark size (FCC 20^3 = 32000 sites)."""
    mb = _lib_or_skip()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=20, sigma=0.02, style="DMD_I")
    s = mb.system_from_workload(w)
    o = Oracle(w)
    check_state(s, o)
    check_forces(s, o, True)


def test_gpu_errors_are_reported(tmp_path):
    mb = _lib_or_skip()
    with pytest.raises(mb.MGError):
        mb.System("LJ")
    w = fx.write_workload(str(tmp_path / "w"), "eam", n=3)
    s = mb.System("EAM")
    s.set_types(["A"], [63.546])
    with pytest.raises(mb.MGError):
        s.force_calc()
    with pytest.raises(mb.MGError) as e:
        s.coef(["ff_coef", "SetFL", str(tmp_path / "missing.eam")])
    assert e.value.code == 2


@pytest.mark.parametrize("kind,kw", [("eam", dict(n=4)), ("dmd", dict(n=4, sigma=0.02, style="DMD_I"))],
                         ids=["eam", "dmd"])
def test_gpu_result_buffers_of_every_kind(tmp_path, kind, kw):
    """force_calc and calc_g copy their per-site result into pageable host
    memory, page-locked host memory or device memory by different routes (a
    side stream beside the reduction for page-locked memory, the main stream
    after it for the others). Each kind of buffer gets its own inputs, so a copy that
    ran before its results were final would return the previous inputs'
    values; each result is compared with a pageable-buffer call on the same
    inputs (to round-off: the sums end in atomics, whose order varies between
    calls), also right after an update_x whose skin test is still pending, and
    also past the skin."""
    mb = _lib_or_skip()
    import torch

    w = fx.write_workload(str(tmp_path / "w"), kind, **kw)
    s = mb.system_from_workload(w)
    N, xd = s.natms, s.x_dim
    x0 = s.get_x()
    rng = np.random.default_rng(5)

    def buffers(cols):
        return [np.zeros((N, cols)), torch.zeros((N, cols), dtype=torch.float64).pin_memory(),
                torch.zeros((N, cols), dtype=torch.float64, device="cuda")]

    def host(a):
        return a if isinstance(a, np.ndarray) else a.cpu().numpy()

    if kind == "dmd":
        # (on the unperturbed lattice: the displacements below bring sites
        # close enough for the rates' exponentials to overflow)
        s.force_calc(1)
        s.create_2nd_neigh_lst()
        s.c_d_calc()
        for g in buffers(s.nt):
            a = rng.normal(0, 0.01, (N, s.nt))
            cost, _ = s.calc_g(a, 0.05, 0, g=g)
            cost_ref, g_ref = s.calc_g(a, 0.05, 0)
            assert np.isfinite(g_ref).all() and np.abs(g_ref).max() > 0
            assert rel(host(g), g_ref) <= TOL
            assert abs(cost - cost_ref) <= TOL * abs(cost_ref)
    for shift in (0.05, 0.7):
        for f in buffers(xd):
            x1 = x0.copy()
            x1[: max(1, N // 10), :3] += rng.normal(0, shift, (max(1, N // 10), 3))
            s.update_x(x1, report=False)
            _, en = s.force_calc(1, f=f)
            f_ref, en_ref = s.force_calc(1)
            assert np.abs(f_ref).max() > 0
            assert rel(host(f), f_ref) <= TOL
            assert rel(en, en_ref) <= TOL


def test_gpu_timing_levels(tmp_path):
    """mg_set_timing: at level 1 (the default) only the whole force call is
    timed and mg_last_time("force.pass1") is an error; level 2 adds the three
    kernels' times, positive and within the call's; level 0 times nothing
    (mg_last_time("force") is an error too). The forces do not change."""
    mb = _lib_or_skip()
    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=4, sigma=0.02, style="DMD_I")
    s = mb.system_from_workload(w)
    f0, _ = s.force_calc(1)
    assert s.last_time("force") > 0
    with pytest.raises(mb.MGError):
        s.last_time("force.pass1")
    s.set_timing(2)
    f1, _ = s.force_calc(1)
    t = [s.last_time(p) for p in ("force.pass1", "force.embed", "force.pass2")]
    assert all(v > 0 for v in t) and sum(t) <= s.last_time("force")
    s.set_timing(0)
    f2, _ = s.force_calc(1)
    for p in ("force", "force.embed"):
        with pytest.raises(mb.MGError):
            s.last_time(p)
    with pytest.raises(mb.MGError):
        s.set_timing(3)
    s.set_timing(1)
    f3, _ = s.force_calc(1)
    assert s.last_time("force") > 0
    for f in (f1, f2, f3):
        assert rel(f, f0) <= TOL
