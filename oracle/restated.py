"""ctypes wrapper around the C restatement oracle (oracle/mapp_oracle.c).

Test infrastructure only: what the GPU library is tested against, never part of it.
``OracleRun`` mirrors the reference harness (oracle/reference.py): it takes a
workload written by ``mapp_b200.fixtures.write_workload`` and reproduces the
reference's call sequence (Min_LBFGS::init order) in the restatement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_mapp.so")
SRC = os.path.join(HERE, "mapp_oracle.c")

STYLES = {"EAM": 0, "FS": 1, "DMD_I": 2, "DMD_II": 3, "DMD": 4}


def build(force=False):
    """Compile the restatement with the reference's arithmetic flags."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB_PATH, SRC, "-lm"])


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.orc_new.restype = P
        L.orc_new.argtypes = [C.c_int, C.c_int]
        L.orc_free.argtypes = [P]
        L.orc_set_tables.argtypes = [P, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, dp, dp, dp]
        L.orc_set_fs.argtypes = [P, dp, dp, dp, dp, dp, dp, dp, dp, ip]
        L.orc_set_dmd.argtypes = [P, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, dp]
        L.orc_set_atoms.argtypes = [P, C.c_int, dp, C.c_double, dp, C.c_void_p, C.c_void_p]
        L.orc_init.argtypes = [P]
        L.orc_update_x.argtypes = [P, dp, C.POINTER(C.c_int)]
        L.orc_update_c.argtypes = [P, dp]
        L.orc_counts.argtypes = [P, ip]
        L.orc_get_x.argtypes = [P, dp]
        L.orc_get_c.argtypes = [P, dp]
        L.orc_get_ghost_src.argtypes = [P, ip]
        L.orc_get_list.argtypes = [P, ip, ip]
        L.orc_get_cutph.argtypes = [P, dp]
        L.orc_get_box.argtypes = [P, dp, dp]
        L.orc_force.argtypes = [P, C.c_int, dp, dp]
        L.orc_energy.argtypes = [P]
        L.orc_energy.restype = C.c_double
        L.orc_create_2nd_neigh_lst.argtypes = [P]
        L.orc_get_crd.argtypes = [P, ip, C.c_void_p, C.c_void_p]
        L.orc_c_d_calc.argtypes = [P, dp]
        L.orc_calc_g.argtypes = [P, C.c_int, C.c_double, dp, dp]
        L.orc_calc_g.restype = C.c_double
        L.orc_get_vec.argtypes = [P, C.c_int, dp]
        L.orc_get_pairs.argtypes = [P, dp]
        L.orc_gauss_hermite.argtypes = [C.c_int, dp, dp]
        L.orc_get_dmd_consts.argtypes = [P, dp]
        L.orc_spline7.argtypes = [C.c_int, C.c_double, dp]
        L.orc_spline9.argtypes = [C.c_int, C.c_double, dp]
        L.orc_lbfgs.argtypes = [P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, dp,
                                C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_lbfgs.restype = C.c_int
        L.orc_cg.argtypes = [P, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, dp, C.POINTER(C.c_int),
                             C.POINTER(C.c_int)]
        L.orc_cg.restype = C.c_int
        L.orc_md_nh.argtypes = [P, dp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                dp, C.c_int, dp]
        L.orc_md_nh.restype = C.c_int
        L.orc_clock_adams.argtypes = [P, C.c_int, C.c_int, C.c_double, dp]
        L.orc_clock_adams.restype = C.c_long
        L.orc_clock_bdf.argtypes = [P, C.POINTER(BdfOpts), dp, C.POINTER(C.c_long)]
        L.orc_clock_bdf.restype = C.c_int
        _lib = L
    return _lib


class BdfOpts(C.Structure):
    """orc_bdf_opts: the options of "clock bdf" (clock_bdf.cpp:14-24 defaults)."""
    _fields_ = [("no_steps", C.c_int), ("max_order", C.c_int), ("max_iter", C.c_int),
                ("min_gamma", C.c_double), ("gamma_red", C.c_double), ("slope", C.c_double),
                ("m_tol", C.c_double), ("a_tol", C.c_double), ("e_tol", C.c_double),
                ("min_del_t", C.c_double), ("max_del_t", C.c_double), ("initial_del_t", C.c_double)]


# Clock_BDF's constructor defaults (clock_bdf.cpp:14-24); the script keyword for
# gamma_red is "red_gamma" (clock_bdf.cpp:46)
BDF_DEFAULTS = dict(max_order=6, max_iter=50, min_gamma=1.0e-10, gamma_red=0.8, slope=0.4, m_tol=1.0e-10,
                    a_tol=1.0e-6, e_tol=0.0, min_del_t=1.0e-12, max_del_t=1.0e4, initial_del_t=-1.0)


def _numbers(lines):
    return np.array([float(t) for ln in lines for t in ln.split("#")[0].split()], dtype=np.float64)


def read_eam_file(path, nt, fs_mode):
    """Raw columns of a setfl / FS table file in the reference's reading order
    (one element header line, ff_eam.cpp:692-775): F [nt][nrho],
    rho [nt][nt][nr] (FS) or [nt][nr] (setfl), r*phi [nt(nt+1)/2][nr]."""
    with open(path) as fp:
        lines = fp.readlines()
    hdr = lines[4].split()
    nrho, drho, nr, dr = int(hdr[0]), float(hdr[1]), int(hdr[2]), float(hdr[3])
    v = _numbers(lines[6:])
    pos = 0
    F = np.zeros((nt, nrho))
    rho = np.zeros((nt, nt, nr)) if fs_mode else np.zeros((nt, nr))
    for i in range(nt):
        F[i] = v[pos:pos + nrho]
        pos += nrho
        if fs_mode:
            for j in range(nt):
                rho[i, j] = v[pos:pos + nr]
                pos += nr
        else:
            rho[i] = v[pos:pos + nr]
            pos += nr
    ncomp = nt * (nt + 1) // 2
    rphi = v[pos:pos + ncomp * nr].reshape(ncomp, nr).copy()
    return dict(nr=nr, dr=dr, nrho=nrho, drho=drho, F=F, rho=rho, rphi=rphi)


def _lagrange4(tab, n_src, d_src, x):
    """The 4-point Lagrange interpolation of ForceField_eam::set_funcfl
    (ff_eam.cpp:565-580): tab holds a leading 0 then the n_src file values,
    the value at grid index m sits at tab[m + 1]."""
    sixth = 1.0 / 6.0
    p = x / d_src + 1.0
    k = int(p)
    k = min(k, n_src - 2)
    k = max(k, 2)
    p -= k
    p = min(p, 2.0)
    c1 = -sixth * p * (p - 1.0) * (p - 2.0)
    c2 = 0.5 * (p * p - 1.0) * (p - 2.0)
    c3 = -0.5 * p * (p + 1.0) * (p - 2.0)
    c4 = sixth * p * (p * p - 1.0)
    return c1 * tab[k - 1] + c2 * tab[k] + c3 * tab[k + 1] + c4 * tab[k + 2]


def read_funcfl_files(paths, nt):
    """ForceField_eam::set_funcfl (ff_eam.cpp:433-670): one single-element
    file per type; the tables are regridded onto nr = int(max_r / max_dr +
    0.5) points of max_dr, and nrho is taken from the same r expression
    (ff_eam.cpp:547-548, so the F grid has nr points too); the pair term is
    27.2 * 0.529 * Z_i Z_j.  Returns the setfl-layout columns (F [nt][nrho],
    rho [nt][nr], r*phi [nt(nt+1)/2][nr]) that the interpolation
    (ForceField_eam::interpolate) then works on.  For more than one type the
    reference stores type i's density in slot i*(i+1) (ff_eam.cpp:583), a slot
    it never allocated; here it is type i's own density, as for setfl."""
    if len(paths) != nt:
        raise ValueError("no of types and number of files should be equal in eam")
    hdr, F0, Z0, R0 = [], [], [], []
    for path in paths:
        with open(path) as fp:
            lines = fp.readlines()
        if len(lines) < 3:
            raise ValueError("eam potential file ended immaturely")
        h = lines[2].split("#")[0].split()
        if len(h) != 5:
            raise ValueError("wrong line in eam file")
        nrho, drho, nr, dr = int(h[0]), float(h[1]), int(h[2]), float(h[3])
        tot = nrho + 2 * nr
        v = []
        for ln in lines[3:]:
            t = ln.split("#")[0].split()
            if len(v) + len(t) > tot:
                raise ValueError("eam potential file ended immaturely")
            v.extend(float(x) for x in t)
            if len(v) == tot:
                break
        if len(v) < tot:
            raise ValueError("eam potential file ended immaturely")
        hdr.append((nrho, drho, nr, dr))
        F0.append([0.0] + v[:nrho])
        Z0.append([0.0] + v[nrho:nrho + nr])
        R0.append([0.0] + v[nrho + nr:])
    maxr = maxrho = maxdr = maxdrho = 0.0
    for nrho, drho, nr, dr in hdr:
        maxr = max(maxr, (nr - 1) * dr)
        maxrho = max(maxrho, (nrho - 1) * drho)
        maxdr = max(maxdr, dr)
        maxdrho = max(maxdrho, drho)
    nr = int(maxr / maxdr + 0.5)
    nrho = int(maxr / maxdr + 0.5)
    dr, drho = maxdr, maxdrho
    F = np.zeros((nt, nrho))
    rho = np.zeros((nt, nr))
    ncomp = nt * (nt + 1) // 2
    rphi = np.zeros((ncomp, nr))
    for i in range(nt):
        for j in range(nrho):
            F[i, j] = _lagrange4(F0[i], hdr[i][0], hdr[i][1], float(j) * drho)
        for j in range(nr):
            rho[i, j] = _lagrange4(R0[i], hdr[i][2], hdr[i][3], float(j) * dr)
    for i in range(nt):
        for j in range(i, nt):
            row = j * (j + 1) // 2 + i
            for m in range(nr):
                r = float(m) * dr
                t0 = _lagrange4(Z0[i], hdr[i][2], hdr[i][3], r)
                t1 = _lagrange4(Z0[j], hdr[j][2], hdr[j][3], r)
                rphi[row, m] = 27.2 * 0.529 * t0 * t1
    return dict(nr=nr, dr=dr, nrho=nrho, drho=drho, F=F, rho=rho, rphi=rphi)


def read_fs_coeffs(path, nt):
    rows = []
    with open(path) as fp:
        for ln in fp:
            t = ln.split("#")[0].split()
            if t:
                rows.append(t)
    rows = rows[1:]
    A = np.array([float(r[0]) for r in rows[:nt]])
    rows = rows[nt:]
    t1 = np.array([float(r[0]) for r in rows[:nt * nt]])
    t2 = np.array([float(r[1]) for r in rows[:nt * nt]])
    rows = rows[nt * nt:]
    ncomp = nt * (nt + 1) // 2
    vals = {}
    k = 0
    for i in range(nt):
        for j in range(i, nt):
            vals[j * (j + 1) // 2 + i] = [float(x) for x in rows[k]]
            k += 1
    arr = np.array([vals[q] for q in range(ncomp)])
    return dict(A=A, t1=t1, t2=t2, cut_rho=arr[:, 0].copy(), cut_phi=arr[:, 1].copy(), k1=arr[:, 2].copy(),
                k2=arr[:, 3].copy(), k3=arr[:, 4].copy(), chk=np.ones(ncomp, dtype=np.int32))


class Oracle:
    """One restated MAPP system (Atoms + Neighbor + ForceField)."""

    def __init__(self, workload: dict):
        L = lib()
        self.w = workload
        cfg = workload["cfg"]
        self.cfg = cfg
        self.style = workload["style"]
        self.nt = len(cfg.names)
        self.dmd = cfg.dmd
        self.h = L.orc_new(STYLES[self.style], self.nt)
        coef = workload["coef"]
        if self.style == "EAM":
            if coef[1] == "FuncFL":
                t = read_funcfl_files(coef[2:], self.nt)
            else:
                t = read_eam_file(coef[2], self.nt, coef[1] == "FS")
            L.orc_set_tables(self.h, t["nr"], t["dr"], t["nrho"], t["drho"], int(coef[1] == "FS"),
                             np.ascontiguousarray(t["F"]), np.ascontiguousarray(t["rho"]), np.ascontiguousarray(t["rphi"]))
        elif self.style == "FS":
            c = read_fs_coeffs(coef[1], self.nt)
            L.orc_set_fs(self.h, c["A"], c["t1"], c["t2"], c["cut_rho"], c["cut_phi"], c["k1"], c["k2"], c["k3"], c["chk"])
        else:
            t = read_eam_file(coef[7], self.nt, coef[6] == "FS")
            L.orc_set_tables(self.h, t["nr"], t["dr"], t["nrho"], t["drho"], int(coef[6] == "FS"),
                             np.ascontiguousarray(t["F"]), np.ascontiguousarray(t["rho"]), np.ascontiguousarray(t["rphi"]))
            L.orc_set_dmd(self.h, float(coef[1]), int(coef[2]), float(coef[3]), float(coef[4]), float(coef[5]),
                          np.asarray(cfg.masses, dtype=np.float64))
        H = np.ascontiguousarray(cfg.H().ravel())
        skin = float(workload.get("skin", 0.5))
        if self.dmd:
            x = np.ascontiguousarray(cfg.x_dmd())
            c = np.ascontiguousarray(cfg.c)
            L.orc_set_atoms(self.h, cfg.natms, H, skin, x, None, c.ctypes.data)
            self._keep = (x, c)
        else:
            from mapp_b200.fixtures import md_order
            order = md_order(cfg)
            s = np.ascontiguousarray(cfg.s[order])
            ty = np.ascontiguousarray(cfg.type[order].astype(np.int32))
            L.orc_set_atoms(self.h, cfg.natms, H, skin, s, ty.ctypes.data, None)
            self._keep = (s, ty)
        L.orc_init(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    @property
    def x_dim(self):
        return 3 + self.nt if self.dmd else 3

    def counts(self):
        out = np.zeros(5, dtype=np.int32)
        lib().orc_counts(self.h, out)
        return dict(natms=int(out[0]), nph=int(out[1]), npairs=int(out[2]), tot_bin=int(out[3]), comm_need=int(out[4]))

    def x_all(self):
        c = self.counts()
        x = np.zeros((c["natms"] + c["nph"]) * self.x_dim)
        lib().orc_get_x(self.h, x)
        return x.reshape(-1, self.x_dim)

    def neighbor_list(self):
        c = self.counts()
        ns = np.zeros(c["natms"], dtype=np.int32)
        fl = np.zeros(max(c["npairs"], 1), dtype=np.int32)
        lib().orc_get_list(self.h, ns, fl)
        return ns, fl[:c["npairs"]]

    def ghost_src(self):
        c = self.counts()
        g = np.zeros(max(c["nph"], 1), dtype=np.int32)
        lib().orc_get_ghost_src(self.h, g)
        return g[:c["nph"]]

    def force(self, st_clc=1):
        c = self.counts()
        f = np.zeros(c["natms"] * self.x_dim)
        en = np.zeros(7)
        lib().orc_force(self.h, st_clc, f, en)
        return f.reshape(-1, self.x_dim), en

    def energy(self):
        return lib().orc_energy(self.h)

    def update_x(self, x):
        r = C.c_int(0)
        lib().orc_update_x(self.h, np.ascontiguousarray(x, dtype=np.float64).ravel(), C.byref(r))
        return r.value

    def update_c(self, c):
        lib().orc_update_c(self.h, np.ascontiguousarray(c, dtype=np.float64).ravel())

    def crd(self):
        lib().orc_create_2nd_neigh_lst(self.h)
        c = self.counts()
        crd = np.zeros(c["natms"] + c["nph"], dtype=np.int32)
        lib().orc_get_crd(self.h, crd, None, None)
        return crd

    def c_d(self):
        c = self.counts()
        out = np.zeros(c["natms"] * self.nt)
        lib().orc_c_d_calc(self.h, out)
        return out.reshape(-1, self.nt)

    def calc_g(self, a, alpha, chk=0):
        c = self.counts()
        g = np.zeros(c["natms"] * self.nt)
        cost = lib().orc_calc_g(self.h, chk, alpha, np.ascontiguousarray(a, dtype=np.float64).ravel(), g)
        return cost, g.reshape(-1, self.nt)

    def vec(self, which):
        c = self.counts()
        n = c["natms"] + c["nph"]
        out = np.zeros(n * (1 if which == 4 else self.nt))
        lib().orc_get_vec(self.h, which, out)
        return out

    def pairs(self):
        c = self.counts()
        nt = self.nt
        n0, n1 = c["npairs"] * nt * nt, c["npairs"] * nt * (nt + 1) // 2
        out = np.zeros(3 * n0 + 3 * n1)
        lib().orc_get_pairs(self.h, out)
        return out

    def lbfgs(self, m=5, max_iter=10000, energy_tol=1e-8, fmax_tol=0.0, max_halvings=0, ls_force_energy=False):
        """Min_LBFGS run (orc_lbfgs): returns dict(code, line_searches, evals,
        energies = force_calc energy after init and after every iteration, x).
        ls_force_energy: line-search energies from the force pass (the batched
        form's rule) instead of energy_calc (the reference's)."""
        e = np.zeros(max_iter + 2)
        err = C.c_int(0)
        nev = C.c_int(0)
        nls = lib().orc_lbfgs(self.h, m, max_iter, energy_tol, fmax_tol, max_halvings, int(ls_force_energy), e,
                              C.byref(err), C.byref(nev))
        x = self.x_all()[: self.counts()["natms"]]
        return {"code": err.value, "line_searches": nls, "evals": nev.value, "energies": e[: nls + 1], "x": x}

    def cg(self, max_iter=10000, energy_tol=1e-8, fmax_tol=0.0, max_halvings=0, ls_force_energy=False):
        """Min_CG run (orc_cg): returns dict(code, line_searches, evals, energies, x) as lbfgs()."""
        e = np.zeros(max_iter + 2)
        err = C.c_int(0)
        nev = C.c_int(0)
        nls = lib().orc_cg(self.h, max_iter, energy_tol, fmax_tol, max_halvings, int(ls_force_energy), e,
                           C.byref(err), C.byref(nev))
        x = self.x_all()[: self.counts()["natms"]]
        return {"code": err.value, "line_searches": nls, "evals": nev.value, "energies": e[: nls + 1], "x": x}

    def md_nh(self, t_tar, t_period, steps, dt, boltz, xd=None, seed=0, eta_iteration=1, eta_chains=3):
        """MD_NH nvt run (orc_md_nh): returns dict(x, xd, energy, virial, ke, t, eta_d)."""
        n = self.counts()["natms"]
        v = np.zeros((n, 3)) if xd is None else np.array(xd, dtype=np.float64).reshape(n, 3).copy()
        mass = np.asarray(self.cfg.masses, dtype=np.float64)
        th = np.zeros(9 + eta_chains)
        rc = lib().orc_md_nh(self.h, mass, t_tar, t_period, eta_iteration, eta_chains, dt, boltz, seed, v.ravel(),
                             steps, th)
        if rc != 0:
            raise ValueError("orc_md_nh rejected the run (zero velocities or chain settings)")
        x = self.x_all()[:n]
        return {"x": x, "xd": v, "energy": th[0], "virial": th[1:7], "ke": th[7], "t": th[8],
                "eta_d": th[9:9 + eta_chains]}

    def clock_adams(self, order, steps, dt):
        """Clock_Adams init + run (orc_clock_adams): returns dict(c, err, n_calc_g)."""
        err = np.zeros(max(steps, 1))
        n = lib().orc_clock_adams(self.h, order, steps, dt, err)
        if n < 0:
            raise ValueError("orc_clock_adams rejected the run (order outside 1..6 or not DMD)")
        c = self.counts()["natms"]
        cc = np.zeros((c + self.counts()["nph"]) * self.nt)
        lib().orc_get_c(self.h, cc)
        return {"c": cc.reshape(-1, self.nt)[:c], "err": err[:steps], "n_calc_g": int(n)}

    def clock_bdf(self, steps, **opts):
        """Clock_BDF init + run (orc_clock_bdf): returns dict(c, n_calc_g, steps,
        del_t, order, t) -- per step the size, the order it ran at and the time
        after it; ``t`` is the final time.  Options as BDF_DEFAULTS."""
        bad = set(opts) - set(BDF_DEFAULTS)
        if bad:
            raise ValueError(f"unknown clock bdf options {sorted(bad)}")
        p = dict(BDF_DEFAULTS, **opts)
        # the constructor's checks (clock_bdf.cpp:29-31, 104-134)
        checks = [(steps <= 0, "no of steps should be greater than zero"),
                  (p["min_gamma"] <= 0.0, "min_gamma should be larger than zero"),
                  (not 0.0 < p["gamma_red"] < 1.0, "gamma_red should be between zero and one"),
                  (not 0.0 < p["slope"] < 1.0, "slope should be between zero and one"),
                  (p["max_iter"] <= 0, "max_iter should be larger than zero"),
                  (p["max_order"] <= 0, "max_order should be larger than zero"),
                  (p["m_tol"] <= 0.0, "m_tol should be larger than zero"),
                  (p["a_tol"] <= 0.0, "a_tol should be larger than zero"),
                  (p["e_tol"] < 0.0, "e_tol should be larger than zero"),
                  (p["min_del_t"] <= 0.0, "min_del_t should be larger than zero"),
                  (p["max_del_t"] <= 0.0, "max_del_t should be larger than zero"),
                  (p["min_del_t"] >= p["max_del_t"], "max_del_t should be larger than min_del_t"),
                  ("initial_del_t" in opts and opts["initial_del_t"] <= 0.0,
                   "initial_del_t should be larger than zero")]
        for bad_opt, msg in checks:
            if bad_opt:
                raise ValueError(msg)
        o = BdfOpts(no_steps=steps, **p)
        hist = np.zeros(3 * max(steps, 1))
        ncg = C.c_long(0)
        rc = lib().orc_clock_bdf(self.h, C.byref(o), hist, C.byref(ncg))
        if rc == -1:
            raise ValueError("c exceeded the domain")
        if rc == -4:
            raise ValueError("the predictor leaves [0, 1] even at min_del_t (the reference would retry for ever)")
        if rc == -3:
            raise ValueError("the step cannot shrink below min_del_t (the reference would retry for ever)")
        if rc < 0:
            raise ValueError("orc_clock_bdf rejected the run (not DMD, or a step-size loop that does not end)")
        c = self.counts()["natms"]
        cc = np.zeros((c + self.counts()["nph"]) * self.nt)
        lib().orc_get_c(self.h, cc)
        h = hist[: 3 * rc].reshape(-1, 3)
        return {"c": cc.reshape(-1, self.nt)[:c], "n_calc_g": int(ncg.value), "steps": rc, "del_t": h[:, 0],
                "order": h[:, 1].astype(int), "t": float(h[-1, 2]) if rc else 0.0}
