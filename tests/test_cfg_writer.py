"""The library's CFG writer (mg_cfg_write_arrays, host code) against the
reference's own WriteCFG (write_cfg.cpp) run by the compiled harness: given
the positions the reference holds after its set-up, the .cfg file (and the
.usr file in DMD mode) agree byte for byte, for cubic and sheared boxes, one
and two species, MD and DMD mode.  The file the writer produces reads back
through the reference-faithful reader to the same box."""
import os

import numpy as np
import pytest

import mapp_b200 as mb
from mapp_b200 import fixtures as fx
from oracle import reference

needs_ref = pytest.mark.skipif(not reference.available(), reason="reference harness not built")
needs_lib = pytest.mark.skipif(not os.path.exists(mb.LIB_PATH), reason="library not built")

CASES = [
    ("eam", dict(n=3, sigma=0.05), None),
    ("eam", dict(n=3, sigma=0.05, nt=2, fmt="FS"), (1.1, -0.7, 0.5)),
    ("dmd", dict(n=3, sigma=0.02, style="DMD_I"), None),
    ("dmd", dict(n=3, sigma=0.02, style="DMD_II"), (0.8, 0.0, -0.6)),
]


@needs_ref
@needs_lib
@pytest.mark.parametrize("kind,kw,tilt", CASES, ids=["eam", "eam2-sheared", "dmd", "dmd-ii-sheared"])
def test_cfg_writer_matches_reference(tmp_path, kind, kw, tilt):
    box = None
    if tilt is not None:
        L = kw["n"] * (3.615 if kind == "eam" else 3.58)
        box = np.array([[L, 0, 0], [tilt[0], L, 0], [tilt[1], tilt[2], L]])
    w = fx.write_workload(str(tmp_path / "w"), kind, box=box, **kw)
    ref_prefix = str(tmp_path / "ref_out")
    rr = reference.RefRun(w, workdir=str(tmp_path / "ref")).dump("s0").writecfg(ref_prefix, 7)
    ref = rr.run()["s0"]
    dmd = kind == "dmd"
    cfg = w["cfg"]
    n = int(ref["meta"]["natms"])
    x_dim = int(ref["meta"]["x_dim"])
    x = ref["x"].reshape(-1, x_dim)[:n]
    H = np.array([[float(v) for v in ref["meta"][f"H{i}"]] for i in range(3)])
    ours = str(tmp_path / "ours")
    if dmd:
        c = ref["c"].reshape(-1, len(cfg.names))[:n]
        path = mb.write_cfg(ours, 7, cfg.names, cfg.masses, H, x, c=c)
    else:
        path = mb.write_cfg(ours, 7, cfg.names, cfg.masses, H, x, type=ref["type"][:n])
    with open(path, "rb") as a, open(ref_prefix + ".00000007.cfg", "rb") as b:
        assert a.read() == b.read()
    if dmd:
        with open(ours + ".00000007.usr", "rb") as a, open(ref_prefix + ".00000007.usr", "rb") as b:
            assert a.read() == b.read()
    back = mb.read_cfg(path, dmd=dmd)
    assert np.allclose(back["H"], H, atol=1e-6)
    assert back["names"] == list(cfg.names)


@needs_lib
def test_cfg_writer_rejects_bad_arguments(tmp_path):
    H = np.diag([10.0, 10.0, 10.0])
    with pytest.raises(mb.MGError):
        mb.write_cfg(str(tmp_path / "a"), 0, ["A"], [1.0], np.zeros((3, 3)), np.zeros((1, 3)), type=[0])
    with pytest.raises(mb.MGError):
        mb.write_cfg(str(tmp_path / "no_such_dir" / "a"), 0, ["A"], [1.0], H, np.zeros((1, 3)), type=[0])
