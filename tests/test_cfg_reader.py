"""The library's CFG reader (mg_cfg_*, host code) against the reference's
ReadCFG: the box it builds and the positions of every site after the
reference's own set-up, bit for bit (through the oracle, which is pinned to
the reference for the same inputs)."""
import os

import numpy as np
import pytest

import mapp_b200 as mb
from mapp_b200 import fixtures as fx
from oracle import reference
from oracle.restated import Oracle

needs_ref = pytest.mark.skipif(not reference.available(), reason="reference harness not built")
needs_lib = pytest.mark.skipif(not os.path.exists(mb.LIB_PATH), reason="library not built")

CASES = [
    ("eam", dict(n=4, sigma=0.05), None),
    ("eam", dict(n=3, sigma=0.05, nt=2, fmt="FS"), None),
    ("eam", dict(n=4, sigma=0.05), (1.3, -0.9, 0.7)),
    ("dmd", dict(n=4, sigma=0.02, style="DMD_I"), (0.8, 0.0, -0.6)),
    ("dmd", dict(n=3, sigma=0.02, style="DMD_II"), None),
]


def _config_from(r, dmd):
    H = r["H"]
    if dmd:
        return fx.Config(float(H[0][0]), r["s"], r["names"], r["masses"], alpha=r["alpha"], c=r["c"], extra={"H": H})
    return fx.Config(float(H[0][0]), r["s"], r["names"], r["masses"], type=r["type"], extra={"H": H})


@needs_ref
@needs_lib
@pytest.mark.parametrize("kind,kw,tilt", CASES, ids=["eam", "eam-2", "eam-sheared", "dmd-sheared", "dmd-ii"])
def test_cfg_reader_matches_reference(tmp_path, kind, kw, tilt):
    box = None
    if tilt is not None:
        L = kw["n"] * (3.615 if kind == "eam" else 3.58)
        box = np.array([[L, 0, 0], [tilt[0], L, 0], [tilt[1], tilt[2], L]])
    w = fx.write_workload(str(tmp_path / "w"), kind, box=box, **kw)
    ref = reference.RefRun(w, workdir=str(tmp_path / "ref")).dump("s0").run()["s0"]
    dmd = kind == "dmd"
    r = mb.read_cfg(w["cfg_path"], dmd=dmd)
    H_ref = np.array([[float(v) for v in ref["meta"][f"H{i}"]] for i in range(3)])
    assert np.array_equal(r["H"], H_ref)
    assert r["names"] == list(w["cfg"].names)
    w2 = dict(w)
    w2["cfg"] = _config_from(r, dmd)
    o = Oracle(w2)
    assert np.array_equal(o.x_all().ravel(), ref["x"])


@needs_ref
@needs_lib
def test_cfg_reader_standard_format_scaled_box(tmp_path):
    """A standard (8-column) CFG with a basic length, a Transform and R, the
    box given with a non-lower-triangular H0: same H and positions.  (The
    reference keeps a file's velocities only when an x_d vector exists before
    the read, which this script does not create; they are compared when the
    dump has them.)"""
    w = fx.write_workload(str(tmp_path / "w"), "eam", n=2)
    rng = np.random.default_rng(3)
    s = rng.uniform(0, 1, (40, 3))
    lines = ["Number of particles = 40", "A = 1.5 Angstrom (basic length-scale)",
             "H0(1,1) = 6.2 A", "H0(1,2) = 0.4 A", "H0(1,3) = 0.0 A",
             "H0(2,1) = 0.3 A", "H0(2,2) = 5.8 A", "H0(2,3) = 0.2 A",
             "H0(3,1) = 0.0 A", "H0(3,2) = -0.5 A", "H0(3,3) = 6.0 A",
             "Transform(1,1) = 1.0", "Transform(2,2) = 1.02", "Transform(3,3) = 0.98",
             "R = 2.0 [ns]"]
    for k in range(40):
        lines.append("%.17g A %.17g %.17g %.17g %.17g %.17g %.17g" % (fx.SPECIES_A.mass, *s[k], *rng.normal(0, 0.01, 3)))
    with open(w["cfg_path"], "w") as fp:
        fp.write("\n".join(lines) + "\n")
    ref = reference.RefRun(w, workdir=str(tmp_path / "ref")).dump("s0").run()["s0"]
    r = mb.read_cfg(w["cfg_path"])
    H_ref = np.array([[float(v) for v in ref["meta"][f"H{i}"]] for i in range(3)])
    assert np.array_equal(r["H"], H_ref)
    assert r["has_velocity"]
    if "xd" in ref:
        assert np.array_equal(r["v"].ravel(), ref["xd"])
    w2 = dict(w)
    w2["cfg"] = _config_from(r, False)
    o = Oracle(w2)
    assert np.array_equal(o.x_all().ravel(), ref["x"])


@needs_lib
def test_cfg_reader_errors(tmp_path):
    bad = tmp_path / "bad.cfg"
    bad.write_text("Number of particles = 1\nthis is not a header line\n")
    with pytest.raises(mb.MGError):
        mb.read_cfg(str(bad))
    with pytest.raises(mb.MGError):
        mb.read_cfg(str(tmp_path / "missing.cfg"))
