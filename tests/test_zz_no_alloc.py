"""The allocation-free entry point mg_fs_energy_noalloc, through the C ABI.

It exists for callers that cannot call cudaMalloc (memory owned by another
allocator, no allocation after start-up, no implicit synchronisation): they
pass their own device buffers and the library uses only its fixed scratch
array.  Checked against the regular ForceField path (mg_ff_energy_calc of an FS
system) on two calls in a row, since every call reuses the same scratch.  The
file name makes pytest collect it last.
"""
import numpy as np
import pytest

from mapp_b200 import fixtures as fx

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _coeffs(path, names, mb):
    from oracle.restated import read_fs_coeffs

    nt = len(names)
    c = read_fs_coeffs(path, nt)
    cf = mb.FsCoeffs()
    cf.ntypes = nt
    for i in range(nt):
        cf.A[i] = c["A"][i]
        for j in range(nt):
            cf.t1[i][j] = c["t1"][i * nt + j]
            cf.t2[i][j] = c["t2"][i * nt + j]
    for q in range(nt * (nt + 1) // 2):
        cf.chk[q] = int(c["chk"][q])
        cf.cut_rho[q] = c["cut_rho"][q]
        cf.cut_phi[q] = c["cut_phi"][q]
        cf.k1[q] = c["k1"][q]
        cf.k2[q] = c["k2"][q]
        cf.k3[q] = c["k3"][q]
    return cf


@pytest.mark.parametrize("nt,n", [(1, 6), (2, 8)])
def test_noalloc_fs_energy_matches_force_field(tmp_path, nt, n):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mapp_b200 as mb

    w = fx.write_workload(str(tmp_path / "w"), "fs", n=n, nt=nt)
    s = mb.system_from_workload(w)
    e_ref = s.energy_calc()
    natms = s.natms
    xo = s.get_x()
    gx, _ = s.ghosts()
    nall = natms + len(gx)
    sizes, pairs = s.neighbor_list()
    order = fx.md_order(w["cfg"])
    typ = w["cfg"].type[order].astype(np.int32)
    _, gown = s.ghosts()
    typ_all = np.concatenate([typ, typ[gown]])
    off = np.zeros(natms + 1, dtype=np.int32)
    off[1:] = np.cumsum(sizes)
    dev = "cuda"
    x_d = torch.from_numpy(np.ascontiguousarray(np.concatenate([xo, gx])[:, :3])).to(dev)
    t_d = torch.from_numpy(typ_all).to(dev)
    o_d = torch.from_numpy(off).to(dev)
    n_d = torch.from_numpy(np.ascontiguousarray(pairs)).to(dev)
    cf = _coeffs(w["coef"][1], w["cfg"].names, mb)
    e_devs = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(2)]
    for call in range(2):
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        e_host = np.zeros(1)
        mb.fs_energy_noalloc(cf, natms, nall, x_d, t_d, o_d, n_d, e_host)
        mb.fs_energy_noalloc(cf, natms, nall, x_d, t_d, o_d, n_d, e_devs[call])
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert abs(e_host[0] - e_ref) <= TOL * abs(e_ref), (call, e_host[0], e_ref)
        assert abs(float(e_devs[call].item()) - e_ref) <= TOL * abs(e_ref), (call, float(e_devs[call].item()), e_ref)
        if call == 1:
            # the second call allocates no device memory (the first may load
            # the library's device code on this device)
            assert free_after == free_before, (free_before, free_after)


def test_noalloc_rejects_oversize_and_host_inputs():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mapp_b200 as mb

    cf = mb.FsCoeffs()
    cf.ntypes = 1
    one_d = torch.zeros(4, dtype=torch.float64, device="cuda")
    one_i = torch.zeros(4, dtype=torch.int32, device="cuda")
    e = np.zeros(1)
    with pytest.raises(mb.MGError) as err:
        mb.fs_energy_noalloc(cf, 2_000_000, 2_000_000, one_d, one_i, one_i, one_i, e)
    assert err.value.code == 6 and "MG_NOALLOC_MAX_ATOMS" in str(err.value)
    with pytest.raises(mb.MGError) as err:
        mb.fs_energy_noalloc(cf, 1, 1, np.zeros(3), one_i, one_i, one_i, e)
    assert err.value.code == 1
