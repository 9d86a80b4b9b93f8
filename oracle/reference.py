"""Runs the compiled reference (oracle/_ref/mapp_ref_harness) on a workload.

Test infrastructure only (the oracle tests the library and is never part of it).  The
harness executable links the unmodified reference objects; see
oracle/ref/harness.cpp for the call sequences it reproduces.  Each run is a
separate process, so a reference abort cannot take the caller down.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "mapp_ref_harness")


def available() -> bool:
    return os.path.exists(HARNESS)


def _meta(path):
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        parts = line.split()
        if not parts:
            continue
        key, vals = parts[0], parts[1:]
        nums = []
        for v in vals:
            try:
                nums.append(int(v))
            except ValueError:
                nums.append(float(v))
        out[key] = nums[0] if len(nums) == 1 else nums
    return out


class RefRun:
    """Builds a command file, runs the harness once and loads every output."""

    def __init__(self, workload: dict, workdir: str | None = None, init: bool = True):
        self.w = workload
        self.dir = workdir or tempfile.mkdtemp(prefix="mapp_ref_")
        os.makedirs(self.dir, exist_ok=True)
        self.lines = [f"script {workload['script']}"]
        style = workload["style"]
        if style.startswith("DMD"):
            self.lines.append(f"oracle_ff {style}")
        else:
            self.lines.append(f"ffcoef_style {style}")
        self.lines.append("ffcoef " + " ".join(workload["coef"]))
        if init:  # Min_LBFGS::init does its own set-up (lbfgs runs pass init=False)
            self.lines.append("init")
        self.steps = []

    def _p(self, tag):
        return os.path.join(self.dir, tag)

    def add(self, line):
        self.lines.append(line)
        return self

    def dump(self, tag="s0"):
        self.steps.append(("dump", tag))
        return self.add(f"dump {self._p(tag)}")

    def force(self, tag="f0", st_clc=1):
        self.steps.append(("force", tag))
        return self.add(f"force {st_clc} {self._p(tag)}")

    def energy(self, tag="e0"):
        self.steps.append(("energy", tag))
        return self.add(f"energy {self._p(tag)}")

    def crd(self, tag="crd"):
        self.steps.append(("crd", tag))
        return self.add(f"crd {self._p(tag)}")

    def cdot(self, tag="cd"):
        self.steps.append(("cdot", tag))
        return self.add(f"cdot {self._p(tag)}")

    def calcg(self, a: np.ndarray, alpha: float, chk=0, tag="g"):
        ap = self._p(tag + ".a.bin")
        np.ascontiguousarray(a, dtype=np.float64).tofile(ap)
        self.steps.append(("calcg", tag))
        return self.add(f"calcg {chk} {alpha!r} {ap} {self._p(tag)}")

    def setx(self, x: np.ndarray, tag="u"):
        xp = self._p(tag + ".x_in.bin")
        np.ascontiguousarray(x, dtype=np.float64).tofile(xp)
        self.steps.append(("setx", tag))
        return self.add(f"setx {xp} {self._p(tag)}")

    def setc(self, c: np.ndarray, tag="c"):
        cp = self._p(tag + ".c_in.bin")
        np.ascontiguousarray(c, dtype=np.float64).tofile(cp)
        return self.add(f"setc {cp}")

    def lbfgs(self, m: int, max_iter: int, energy_tol: float, tag="lb"):
        """The reference Min_LBFGS: init, run, fin (construct with init=False)."""
        self.steps.append(("lbfgs", tag))
        return self.add(f"lbfgs {m} {max_iter} {energy_tol!r} {self._p(tag)}")

    def cg(self, max_iter: int, energy_tol: float, tag="cg"):
        """The reference Min_CG: init, run, fin (construct with init=False)."""
        self.steps.append(("cg", tag))
        return self.add(f"cg {max_iter} {energy_tol!r} {self._p(tag)}")

    def writecfg(self, prefix: str, step: int = 0):
        """The reference WriteCFG's file of the current state (x, and c in DMD mode)."""
        return self.add(f"writecfg {prefix} {step}")

    def adams(self, order: int, steps: int, dt: float, tag="adams"):
        """The reference Clock_Adams: init, run, fin (construct with init=False)."""
        self.steps.append(("adams", tag))
        return self.add(f"adams {order} {steps} {dt!r} {self._p(tag)}")

    def bdf(self, steps: int, tag="bdf", **opts):
        """The reference Clock_BDF "clock bdf steps [key value ...]": init, run,
        fin (construct with init=False).  Option keys as in the reference's
        script (gamma_red is spelled red_gamma there)."""
        self.steps.append(("bdf", tag))
        def text(v):
            return str(int(v)) if isinstance(v, (int, np.integer)) else repr(float(v))

        kv = " ".join(f"{'red_gamma' if k == 'gamma_red' else k} {text(v)}" for k, v in opts.items())
        return self.add(f"bdf {steps} {self._p(tag)} {kv}")

    def md(self, t_tar: float, t_period: float, steps: int, dt: float, boltz: float, xd=None, seed=0,
           eta_iteration=1, eta_chains=3, tag="md"):
        """The reference MD_NH nvt run (construct with init=False): velocities
        ``xd`` [natms][3] in the reader's atom order, or create_vel with ``seed``."""
        xp = "-"
        if xd is not None:
            xp = self._p(tag + ".xd_in.bin")
            np.ascontiguousarray(xd, dtype=np.float64).tofile(xp)
        self.steps.append(("md", tag))
        return self.add(f"md {t_tar!r} {t_period!r} {eta_iteration} {eta_chains} {dt!r} {boltz!r} {seed} {steps} "
                        f"{xp} {self._p(tag)}")

    def time(self, what: str, reps: int, tag="t"):
        self.steps.append(("time", tag))
        return self.add(f"time {what} {reps} {self._p(tag)}")

    def run(self, timeout=600) -> dict:
        cmd_path = self._p("commands.txt")
        lines = []
        for ln in self.lines:
            if ln.startswith("ffcoef_style "):
                # EAM / FS use the stock reference classes: create them by script
                continue
            lines.append(ln)
        style = self.w["style"]
        if not style.startswith("DMD"):
            # stock style: create the force field with the reference's own "ff" command
            script2 = self._p("in_stock.mapp")
            with open(self.w["script"]) as src, open(script2, "w") as dst:
                dst.write(src.read())
                dst.write(f"ff {style}\n")
                dst.write(" ".join(self.w["coef"]) + "\n")
            lines = [f"script {script2}"] + [ln for ln in lines[1:] if not ln.startswith("ffcoef ")]
        with open(cmd_path, "w") as fp:
            fp.write("\n".join(lines) + "\n")
        proc = subprocess.run([HARNESS, cmd_path], capture_output=True, text=True, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"reference harness failed ({proc.returncode}):\n{proc.stdout[-2000:]}\n{proc.stderr[-2000:]}")
        self.stdout = proc.stdout
        return self.load()

    def load(self) -> dict:
        res = {}
        for kind, tag in self.steps:
            p = self._p(tag)
            m = _meta(p + ".meta")
            d = {"meta": m}
            for fn in os.listdir(self.dir):
                if fn.startswith(tag + ".") and fn.endswith(".bin") and not fn.endswith("_in.bin") and not fn.endswith(".a.bin"):
                    name = fn[len(tag) + 1:-4]
                    dt = np.int32 if name in ("nsize", "nlist", "type", "id", "crd") else np.float64
                    d[name] = np.fromfile(os.path.join(self.dir, fn), dtype=dt)
            res[tag] = d
        return res
