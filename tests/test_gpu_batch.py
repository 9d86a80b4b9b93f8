"""Batched form: independent DMD cells relaxed by L-BFGS together on the GPU,
checked cell by cell against the oracle's restatement of Min_LBFGS::run +
LineSearch_BackTrack::line_min (orc_lbfgs, pinned to the reference in
tests/test_oracle_lbfgs.py) with line-search energies from the force pass."""
import tempfile

import numpy as np
import pytest

from mapp_b200 import fixtures as fx

pytestmark = pytest.mark.gpu

SHAPES = [(3, 3, 3), (3, 3, 2), (4, 4, 4), (5, 5, 3)]


def _mb():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mapp_b200

    return mapp_b200


def _builder(mb):
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=2, style="DMD_I")
    return mb.system_from_workload(w)


def _cells():
    return [fx.make_dmd_cell(*sh, sigma=0.03, seed=10 + k, mean_cA=0.3 + 0.1 * k) for k, sh in enumerate(SHAPES)]


def _oracle_run(cfg, max_iter, fmax_tol, energy_tol, max_halvings):
    from oracle.restated import Oracle

    w = fx.write_workload(tempfile.mkdtemp(), "dmd", cfg=cfg, style="DMD_I")
    o = Oracle(w)
    r = o.lbfgs(5, max_iter, energy_tol, fmax_tol=fmax_tol, max_halvings=max_halvings, ls_force_energy=True)
    f, _ = o.force(1)
    return r, f


def test_batch_fp64_matches_oracle_per_cell():
    mb = _mb()
    b0 = _builder(mb)
    cells = _cells()
    B = mb.Batch(b0)
    for c in cells:
        B.add_cell(c)
    B.set_params(5, 200, 1e-5, 1e-8, 60)
    st = B.relax()
    assert st["iterations"] > 0 and st["evaluations"] >= len(cells)
    for k, c in enumerate(cells):
        x, f, r = B.cell_result(k)
        ro, fo = _oracle_run(c, 200, 1e-5, 1e-8, 60)
        e_ref = ro["energies"][-1]
        # A stalled cell's last line search ends on the energy tolerance (it
        # accepts a step that lowers the energy by less than 1e-8) or on the
        # step limit; which of the two depends on the last bits of energies
        # that the GPU sums in another order, so either is taken for the other.
        assert r["code"] == ro["code"] or {r["code"], ro["code"]} <= {3, 5}, (k, r, ro["code"])
        assert r["iterations"] == ro["line_searches"] - 1
        assert abs(r["energy"] - e_ref) <= 1e-12 * abs(e_ref)
        # trajectories of a dozen iterations, summed in another order: positions
        # within 1e-9 A, forces within 1e-7 of their largest component
        assert np.max(np.abs(x - ro["x"])) <= 1e-9
        assert np.max(np.abs(f - fo)) <= 1e-7 * np.max(np.abs(fo))
        assert r["t_ms"] > 0


def test_batch_skin_rebuilds_keep_the_trajectory():
    """A tiny skin makes trial points leave the lists: the device loop pauses,
    the host rebuilds every cell, and the result still follows the oracle
    (which rebuilds inside update_0 at the same points)."""
    mb = _mb()
    w = fx.write_workload(tempfile.mkdtemp(), "dmd", n=2, style="DMD_I", skin=0.02)
    b0 = mb.system_from_workload(w, skin=0.02)
    cells = _cells()[:2]
    B = mb.Batch(b0)
    for c in cells:
        B.add_cell(c)
    B.set_params(5, 40, 0.0, 1e-8, 60)
    st = B.relax()
    assert st["rebuild_rounds"] >= 1
    from oracle.restated import Oracle

    for k, c in enumerate(cells):
        x, f, r = B.cell_result(k)
        wc = fx.write_workload(tempfile.mkdtemp(), "dmd", cfg=c, style="DMD_I", skin=0.02)
        o = Oracle(wc)
        ro = o.lbfgs(5, 40, 1e-8, fmax_tol=0.0, max_halvings=60, ls_force_energy=True)
        assert r["code"] == ro["code"] or {r["code"], ro["code"]} <= {3, 5}
        assert abs(r["energy"] - ro["energies"][-1]) <= 1e-11 * abs(ro["energies"][-1])


def test_batch_fp32_form_and_tuning_cache(tmp_path):
    mb = _mb()
    b0 = _builder(mb)
    cells = fx.make_batch_cells(24, seed=3, lo=500, hi=3000)
    cache = tmp_path / "tune.txt"
    results = {}
    for form in (mb.MG_FORM_FP64, mb.MG_FORM_FP32):
        B = mb.Batch(b0)
        for c in cells:
            B.add_cell(c)
        B.set_params(5, 50, 1e-5, 1e-8, 60)
        B.set_form(form)
        B.set_tuning(True, cache)
        st = B.relax()
        assert st["from_cache"] == 0 and st["bps1"] > 0 and st["lbfgs_threads"] in (128, 256, 512, 1024)
        results[form] = [B.cell_result(k)[2] for k in range(len(cells))]
        B.close()
        # a new batch of the same shape takes its launch shapes from the cache
        B2 = mb.Batch(b0)
        for c in cells:
            B2.add_cell(c)
        B2.set_params(5, 50, 1e-5, 1e-8, 60)
        B2.set_form(form)
        B2.set_tuning(True, cache)
        st2 = B2.relax()
        assert st2["from_cache"] == 1 and st2["tune_ms"] == 0.0
        assert (st2["bps1"], st2["bps2"], st2["lbfgs_threads"]) == (st["bps1"], st["bps2"], st["lbfgs_threads"])
        B2.close()
    assert cache.read_text().count("\n") == 2
    e64 = np.array([r["energy"] for r in results[mb.MG_FORM_FP64]])
    e32 = np.array([r["energy"] for r in results[mb.MG_FORM_FP32]])
    n = np.array([r["natms"] for r in results[mb.MG_FORM_FP64]])
    # the FP32 form follows its own (noisier) path; the free energies it reaches
    # agree with the FP64 ones to a few meV per cell
    assert np.all(np.abs(e32 - e64) / n < 1e-3)
    assert all(r["code"] in (1, 3, 4, 5) for r in results[mb.MG_FORM_FP32])


@pytest.mark.parametrize("threads,cluster", [(128, 2), (128, 4), (64, 16)])
def test_batch_cluster_steps_match_oracle(threads, cluster):
    """The L-BFGS step of a cell spread over a thread-block cluster (CTAs
    share the cell's vectors, reductions through distributed shared memory)
    follows the same trajectories."""
    mb = _mb()
    b0 = _builder(mb)
    cells = _cells()
    B = mb.Batch(b0)
    for c in cells:
        B.add_cell(c)
    B.set_params(5, 200, 1e-5, 1e-8, 60)
    B.set_launch(0, 0, threads, cluster)
    st = B.relax()
    assert st["lbfgs_cluster"] == cluster and st["lbfgs_threads"] == threads
    for k, c in enumerate(cells):
        x, f, r = B.cell_result(k)
        ro, fo = _oracle_run(c, 200, 1e-5, 1e-8, 60)
        e_ref = ro["energies"][-1]
        assert r["code"] == ro["code"] or {r["code"], ro["code"]} <= {3, 5}, (k, r, ro["code"])
        assert r["iterations"] == ro["line_searches"] - 1
        assert abs(r["energy"] - e_ref) <= 1e-12 * abs(e_ref)
        assert np.max(np.abs(x - ro["x"])) <= 1e-9


def test_min_lbfgs_single_system_matches_oracle(tmp_path):
    """mg_min_lbfgs: the system relaxes itself on the device (one cell, its
    step on a 16-CTA cluster) and holds the final state afterwards."""
    mb = _mb()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=6, sigma=0.03, style="DMD_I")
    s = mb.system_from_workload(w)
    r, st = s.min_lbfgs(5, 60, 1e-5, 1e-8, 60, cluster=16)
    assert st["lbfgs_cluster"] == 16
    o = Oracle(w)
    ro = o.lbfgs(5, 60, 1e-8, fmax_tol=1e-5, max_halvings=60, ls_force_energy=True)
    e_ref = ro["energies"][-1]
    assert r["code"] == ro["code"] or {r["code"], ro["code"]} <= {3, 5}
    assert r["iterations"] == ro["line_searches"] - 1
    assert abs(r["energy"] - e_ref) <= 1e-12 * abs(e_ref)
    # the system now holds the relaxed state (positions wrapped into the box,
    # as a list rebuild does): equal up to box vectors
    L = w["cfg"].L
    x = s.get_x()
    dx = x - ro["x"]
    dx[:, :3] -= L * np.round(dx[:, :3] / L)
    assert np.max(np.abs(dx)) <= 1e-9
    # Its own force call agrees with the oracle rebuilt at that state.  (Not
    # with the oracle's last step: for two species the reference's pair energy
    # takes the cross-species phi with alpha_i[a], alpha_j[b] for the order the
    # half list names the pair in, so re-wrapping sites changes the energy.)
    o2 = Oracle(w)
    far = x.copy()
    far[:, :3] += 0.9  # beyond the skin: update_0 rebuilds, then the state itself
    o2.update_x(far)
    o2.update_x(x)
    f, en = s.force_calc(1)
    fo, eno = o2.force(1)
    assert abs(en[0] - eno[0]) <= 1e-10 * abs(eno[0])
    assert np.max(np.abs(f - fo)) <= 1e-9 * np.max(np.abs(fo))


def test_batch_cg_matches_oracle_per_cell():
    """The batched form with Min_CG's Polak-Ribiere direction, cell by cell
    against orc_cg (pinned to the reference's Min_CG).  Over the first 8
    iterations, while the energy still falls by far more than its rounding,
    every cell follows the oracle's trajectory (positions within 1e-9 A).
    Later, as a cell stalls, an Armijo test or the energy tolerance can fall
    within the last bits of energies the GPU sums in another order, and the
    two runs may stop a few iterations apart; the full runs are then compared
    by their stop reason and final energy (1e-8 relative)."""
    from oracle.restated import Oracle

    mb = _mb()
    b0 = _builder(mb)
    cells = _cells()

    def relax(max_iter, fmax_tol, energy_tol):
        B = mb.Batch(b0)
        for c in cells:
            B.add_cell(c)
        B.set_params(5, max_iter, fmax_tol, energy_tol, 60)
        B.set_method(mb.MG_MIN_CG)
        B.relax()
        return B

    B = relax(8, 0.0, 1e-12)
    for k, c in enumerate(cells):
        x, f, r = B.cell_result(k)
        w = fx.write_workload(tempfile.mkdtemp(), "dmd", cfg=c, style="DMD_I")
        o = Oracle(w)
        ro = o.cg(8, 1e-12, fmax_tol=0.0, max_halvings=60, ls_force_energy=True)
        fo, _ = o.force(1)
        e_ref = ro["energies"][-1]
        assert r["code"] == ro["code"], (k, r, ro["code"])
        assert r["iterations"] == ro["line_searches"] - 1
        assert abs(r["energy"] - e_ref) <= 1e-12 * abs(e_ref)
        assert np.max(np.abs(x - ro["x"])) <= 1e-9
        assert np.max(np.abs(f - fo)) <= 1e-7 * np.max(np.abs(fo))
    B.close()
    B = relax(200, 1e-5, 1e-8)
    for k, c in enumerate(cells):
        x, f, r = B.cell_result(k)
        w = fx.write_workload(tempfile.mkdtemp(), "dmd", cfg=c, style="DMD_I")
        ro = Oracle(w).cg(200, 1e-8, fmax_tol=1e-5, max_halvings=60, ls_force_energy=True)
        e_ref = ro["energies"][-1]
        assert {r["code"], ro["code"]} <= {3, 5}, (k, r, ro["code"])
        # stalled runs that stopped a few iterations apart: energies within
        # 1e-8 relative (the last iterations of a stall lower the energy by
        # about 1e-7 eV each)
        assert abs(r["energy"] - e_ref) <= 1e-8 * abs(e_ref)


def test_min_cg_single_system_matches_oracle(tmp_path):
    """mg_min_cg: the system relaxes itself by conjugate gradient on the
    device (one cell, its step on a 4-CTA cluster)."""
    mb = _mb()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=6, sigma=0.03, style="DMD_I")
    s = mb.system_from_workload(w)
    r, st = s.min_cg(60, 1e-5, 1e-8, 60, cluster=4)
    assert st["lbfgs_cluster"] == 4
    ro = Oracle(w).cg(60, 1e-8, fmax_tol=1e-5, max_halvings=60, ls_force_energy=True)
    e_ref = ro["energies"][-1]
    assert r["code"] == ro["code"] or {r["code"], ro["code"]} <= {3, 5}
    assert r["iterations"] == ro["line_searches"] - 1
    assert abs(r["energy"] - e_ref) <= 1e-12 * abs(e_ref)
    L = w["cfg"].L
    dx = s.get_x() - ro["x"]
    dx[:, :3] -= L * np.round(dx[:, :3] / L)
    assert np.max(np.abs(dx)) <= 1e-9


@pytest.mark.parametrize("method", ["lbfgs", "cg"])
def test_single_system_step_on_the_whole_gpu(tmp_path, method):
    """The one-cell step on every SM (MG_LAUNCH_WHOLE_GPU: cooperative launch,
    grid barriers, reductions in CTA order) follows the oracle like the
    cluster step does."""
    mb = _mb()
    from oracle.restated import Oracle

    w = fx.write_workload(str(tmp_path / "w"), "dmd", n=6, sigma=0.03, style="DMD_I")
    s = mb.system_from_workload(w)
    o = Oracle(w)
    if method == "lbfgs":
        r, st = s.min_lbfgs(5, 8, 0.0, 1e-12, 60, cluster=mb.MG_LAUNCH_WHOLE_GPU)
        ro = o.lbfgs(5, 8, 1e-12, fmax_tol=0.0, max_halvings=60, ls_force_energy=True)
    else:
        r, st = s.min_cg(8, 0.0, 1e-12, 60, cluster=mb.MG_LAUNCH_WHOLE_GPU)
        ro = o.cg(8, 1e-12, fmax_tol=0.0, max_halvings=60, ls_force_energy=True)
    assert st["lbfgs_cluster"] == mb.MG_LAUNCH_WHOLE_GPU
    e_ref = ro["energies"][-1]
    assert r["code"] == ro["code"]
    assert r["iterations"] == ro["line_searches"] - 1
    assert abs(r["energy"] - e_ref) <= 1e-12 * abs(e_ref)
    L = w["cfg"].L
    dx = s.get_x() - ro["x"]
    dx[:, :3] -= L * np.round(dx[:, :3] / L)
    assert np.max(np.abs(dx)) <= 1e-9
