"""Seeded synthetic workloads in MAPP's own on-disk formats.

Writes the three inputs MAPP's hot path consumes, byte-for-byte readable by
both the reference and this package:

* extended CFG configurations (``read_cfg.cpp:236-358`` header,
  ``read_cfg.cpp:562-627`` DMD atom lines ``s0 s1 s2 alpha_1..alpha_n c_1..c_n``);
* tabulated EAM potentials in setfl / Finnis-Sinclair layout
  (``ff_eam.cpp:674-879``, ``ff_eam.cpp:883-1108``, ``ff_dmd_I.cpp:1300-1548``:
  three comment lines, an element line, ``Nrho drho Nr dr cut``, ONE element
  header line for all species, then 5 values per line);
* the analytic Finnis-Sinclair coefficient file (``ff_fs.cpp:113-335``).

Potentials follow the synthetic species defined for the benchmark workloads:
species A  phi = 0.35 exp(-8 (r/2.556 - 1)),  rho = exp(-4 (r/2.556 - 1)),
F = -1.8 sqrt(rho); species B  phi prefactor 0.40, r_e = 2.49, exponents
8.4 / 4.2, F = -2.0 sqrt(rho); the A-B cross pair uses the geometric-mean
prefactor and arithmetic-mean r_e and exponents for both phi and rho
(rho_AB = rho_BA).  Every pair function is multiplied by the quintic
smoothstep taper S(t) = 1 - (10t^3 - 15t^4 + 6t^5), t = (r - 4.5) / 0.5
clamped to [0, 1], so it vanishes at the 5 A cut.

All values are written with 17 significant digits, so a reader that parses
with strtod/atof recovers exactly the doubles generated here.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

#: amu masses used for the two synthetic species (not set by the workload
#: definitions; these are the Cu and Ni values)
MASS_A = 63.546
MASS_B = 58.693

R_CUT = 5.0
TAPER_ON = 4.5
NR = 10000
NRHO = 10000
RHO_MAX = 40.0


@dataclass(frozen=True)
class Species:
    name: str
    mass: float
    phi0: float
    re: float
    beta_phi: float
    beta_rho: float
    f0: float


SPECIES_A = Species("A", MASS_A, 0.35, 2.556, 8.0, 4.0, 1.8)
SPECIES_B = Species("B", MASS_B, 0.40, 2.49, 8.4, 4.2, 2.0)
# extra synthetic species for multi-component tests (not part of any benchmark workload)
SPECIES_C = Species("C", 55.845, 0.38, 2.52, 8.2, 4.1, 1.9)
SPECIES_D = Species("D", 58.933, 0.36, 2.54, 8.1, 4.05, 1.85)
ALL_SPECIES = (SPECIES_A, SPECIES_B, SPECIES_C, SPECIES_D)


def taper(r: np.ndarray) -> np.ndarray:
    t = np.clip((r - TAPER_ON) / (R_CUT - TAPER_ON), 0.0, 1.0)
    return 1.0 - (10.0 * t**3 - 15.0 * t**4 + 6.0 * t**5)


def pair_phi(r, phi0, re, beta):
    return phi0 * np.exp(-beta * (r / re - 1.0)) * taper(r)


def pair_rho(r, re, beta):
    return np.exp(-beta * (r / re - 1.0)) * taper(r)


def cross(a: Species, b: Species):
    """Cross-pair parameters: geometric-mean prefactor, arithmetic means otherwise."""
    return (math.sqrt(a.phi0 * b.phi0), 0.5 * (a.re + b.re),
            0.5 * (a.beta_phi + b.beta_phi), 0.5 * (a.beta_rho + b.beta_rho))


@dataclass
class EamTables:
    """Raw tabulated columns exactly as a setfl / FS file stores them."""

    names: list
    masses: list
    nr: int
    dr: float
    nrho: int
    drho: float
    F: np.ndarray        # [nt][nrho]
    rho: np.ndarray      # [nt][nt][nr]  (block [i][j] of the FS layout)
    rphi: np.ndarray     # [nt(nt+1)/2][nr] in COMP order (i >= j, row i*(i+1)/2 + j)


def make_tables(species=(SPECIES_A,), nr=NR, nrho=NRHO, rho_max=RHO_MAX) -> EamTables:
    nt = len(species)
    dr = R_CUT / (nr - 1)
    drho = rho_max / (nrho - 1)
    r = np.arange(nr, dtype=np.float64) * dr
    rh = np.arange(nrho, dtype=np.float64) * drho
    F = np.stack([-s.f0 * np.sqrt(rh) for s in species])
    rho = np.zeros((nt, nt, nr))
    rphi = np.zeros((nt * (nt + 1) // 2, nr))
    for i, si in enumerate(species):
        for j, sj in enumerate(species):
            if i == j:
                rho[i, j] = pair_rho(r, si.re, si.beta_rho)
            else:
                _, re, _, brho = cross(si, sj)
                rho[i, j] = pair_rho(r, re, brho)
        for j in range(i + 1):
            sj = species[j]
            if i == j:
                phi = pair_phi(r, si.phi0, si.re, si.beta_phi)
            else:
                p0, re, bphi, _ = cross(si, sj)
                phi = pair_phi(r, p0, re, bphi)
            rphi[i * (i + 1) // 2 + j] = r * phi
    return EamTables([s.name for s in species], [s.mass for s in species],
                     nr, dr, nrho, drho, F, rho, rphi)


def _write_values(fp, values):
    v = np.asarray(values, dtype=np.float64).ravel()
    n5 = (len(v) // 5) * 5
    for k in range(0, n5, 5):
        fp.write("%.17g %.17g %.17g %.17g %.17g\n" % tuple(v[k:k + 5]))
    if n5 < len(v):
        fp.write(" ".join("%.17g" % x for x in v[n5:]) + "\n")


def _header(fp, t: EamTables):
    fp.write("# synthetic EAM tables generated by mapp_b200.fixtures\n")
    fp.write("# species: %s\n" % " ".join(t.names))
    fp.write("# cut %.6f A, taper from %.2f A\n" % (R_CUT, TAPER_ON))
    fp.write("%d %s\n" % (len(t.names), " ".join(t.names)))
    fp.write("%d %.17g %d %.17g %.17g\n" % (t.nrho, t.drho, t.nr, t.dr, R_CUT))
    # one element header line for all species: the reference readers read
    # exactly one such line (ff_eam.cpp:770, ff_dmd_I.cpp:1397)
    fp.write("0 %.17g 0 fcc\n" % t.masses[0])


def write_setfl(path: str, t: EamTables):
    """setfl layout: per element F then rho_element, then r*phi for i >= j."""
    with open(path, "w") as fp:
        _header(fp, t)
        nt = len(t.names)
        for i in range(nt):
            _write_values(fp, t.F[i])
            _write_values(fp, t.rho[i, i])
        for row in t.rphi:
            _write_values(fp, row)


def write_fs(path: str, t: EamTables):
    """Finnis-Sinclair layout: per element F then rho blocks [i][0..nt), then r*phi."""
    with open(path, "w") as fp:
        _header(fp, t)
        nt = len(t.names)
        for i in range(nt):
            _write_values(fp, t.F[i])
            for j in range(nt):
                _write_values(fp, t.rho[i, j])
        for row in t.rphi:
            _write_values(fp, row)


# funcfl grid: deliberately not the setfl one, so that the reference's
# regridding onto nr - 1 points (and nrho taken from the r grid) is exercised
FUNCFL_NR = 2500
FUNCFL_NRHO = 2000
FUNCFL_RHO_MAX = 40.0
ZCONST = 27.2 * 0.529  # eV A: r*phi = ZCONST * Z_i(r) Z_j(r) in the funcfl convention


def write_funcfl(path: str, sp: "Species", nr=FUNCFL_NR, nrho=FUNCFL_NRHO, rho_max=FUNCFL_RHO_MAX):
    """One single-element funcfl file: a comment line; "Z mass a lattice";
    "nrho drho nr dr cut"; then F(rho) on nrho points, the effective charge
    Z(r) and rho(r) on nr points.  Z(r) = sqrt(r phi(r) / ZCONST), so that the
    pair term the reader forms, ZCONST Z_i Z_j, is r*phi for like pairs (phi
    is positive for these species)."""
    dr = R_CUT / (nr - 1)
    drho = rho_max / (nrho - 1)
    r = np.arange(nr, dtype=np.float64) * dr
    rh = np.arange(nrho, dtype=np.float64) * drho
    F = -sp.f0 * np.sqrt(rh)
    z = np.sqrt(np.maximum(r * pair_phi(r, sp.phi0, sp.re, sp.beta_phi), 0.0) / ZCONST)
    rho = pair_rho(r, sp.re, sp.beta_rho)
    with open(path, "w") as fp:
        fp.write("# synthetic funcfl table for species %s generated by mapp_b200.fixtures\n" % sp.name)
        fp.write("29 %.17g 3.615 fcc\n" % sp.mass)
        fp.write("%d %.17g %d %.17g %.17g\n" % (nrho, drho, nr, dr, R_CUT))
        _write_values(fp, F)
        _write_values(fp, z)
        _write_values(fp, rho)


@dataclass
class FsCoeffs:
    """Analytic Finnis-Sinclair coefficients (ff_fs.cpp:14-21 functional form)."""

    names: list
    masses: list
    A: list
    t1: list       # [nt][nt]
    t2: list
    cut_rho: list  # COMP order
    cut_phi: list
    k1: list
    k2: list
    k3: list


def make_fs_coeffs(nt=1) -> FsCoeffs:
    names = ["A", "B"][:nt]
    masses = [MASS_A, MASS_B][:nt]
    A = [1.5, 2.2][:nt]
    t1 = [[1.0, 0.9], [1.1, 0.8]]
    t2 = [[0.3, 0.25], [0.35, 0.2]]
    t1 = [row[:nt] for row in t1[:nt]]
    t2 = [row[:nt] for row in t2[:nt]]
    ncomp = nt * (nt + 1) // 2
    cut_rho = [3.8, 3.7, 3.6][:ncomp]
    cut_phi = [3.5, 3.45, 3.4][:ncomp]
    k1 = [1.1, 1.3, 0.9][:ncomp]
    k2 = [-0.30, -0.35, -0.25][:ncomp]
    k3 = [-0.03, -0.02, -0.04][:ncomp]
    return FsCoeffs(names, masses, A, t1, t2, cut_rho, cut_phi, k1, k2, k3)


def write_fs_coeffs(path: str, c: FsCoeffs):
    nt = len(c.names)
    with open(path, "w") as fp:
        fp.write("# analytic Finnis-Sinclair coefficients (synthetic)\n")
        fp.write(" ".join(c.names) + "\n")
        fp.write("# A per type\n")
        for a in c.A:
            fp.write("%.17g\n" % a)
        fp.write("# t_1 t_2 per ordered type pair\n")
        for i in range(nt):
            for j in range(nt):
                fp.write("%.17g %.17g\n" % (c.t1[i][j], c.t2[i][j]))
        fp.write("# r_cut_rho r_cut_phi k_1 k_2 k_3 per unordered pair\n")
        k = 0
        for i in range(nt):
            for j in range(i, nt):
                comp = j * (j + 1) // 2 + i  # COMP(i, j) with i <= j
                fp.write("%.17g %.17g %.17g %.17g %.17g\n" % (
                    c.cut_rho[comp], c.cut_phi[comp], c.k1[comp], c.k2[comp], c.k3[comp]))
                k += 1


@dataclass
class Config:
    """One periodic configuration in the state a CFG read leaves behind."""

    L: float                 # cubic box edge (H = diag(L))
    s: np.ndarray            # [N][3] fractional positions in [0, 1)
    names: list
    masses: list
    type: np.ndarray | None = None   # [N] species index (MD mode)
    alpha: np.ndarray | None = None  # [N][nt] Gaussian exponents (DMD mode)
    c: np.ndarray | None = None      # [N][nt] concentrations (DMD mode)
    extra: dict = field(default_factory=dict)

    @property
    def natms(self):
        return self.s.shape[0]

    @property
    def dmd(self):
        return self.alpha is not None

    def H(self) -> np.ndarray:
        if "H" in self.extra:
            return np.array(self.extra["H"], dtype=np.float64)
        return np.diag([self.L, self.L, self.L]).astype(np.float64)

    def x_dmd(self) -> np.ndarray:
        """Owned x vector in the reference's DMD layout [s0 s1 s2 alpha...]."""
        return np.ascontiguousarray(np.concatenate([self.s, self.alpha], axis=1))


def fcc_sites(n: int, a: float) -> np.ndarray:
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)
    g = np.arange(n, dtype=np.float64)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    return ((cells[:, None, :] + base[None, :, :]).reshape(-1, 3)) * a


def fcc_box(nx: int, ny: int, nz: int, a: float) -> np.ndarray:
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), axis=-1)
    cells = g.reshape(-1, 3).astype(np.float64)
    return ((cells[:, None, :] + base[None, :, :]).reshape(-1, 3)) * a


def _wrap(s: np.ndarray) -> np.ndarray:
    s = s - np.floor(s)
    s[s >= 1.0] = 0.0
    return s


def make_md_config(n=10, a=3.615, sigma=0.05, seed=1234, nt=1) -> Config:
    """FCC n^3 cells displaced by a seeded Gaussian (EAM / FS workloads)."""
    rng = np.random.default_rng(seed)
    x = fcc_sites(n, a) + rng.normal(0.0, sigma, size=(4 * n**3, 3))
    L = n * a
    s = _wrap(x / L)
    typ = np.zeros(len(s), dtype=np.int32)
    if nt > 1:
        typ = rng.integers(0, nt, size=len(s)).astype(np.int32)
    return Config(L, s, ["A", "B"][:nt], [MASS_A, MASS_B][:nt], type=typ)


def make_dmd_config(n=20, a=3.58, sigma=0.0, seed=4321, nt=2,
                    w_lo=0.08, w_hi=0.15, mean_cA=None) -> Config:
    """FCC n^3 DMD sites: alpha = 1/w^2 with w ~ U(w_lo, w_hi) A per site and
    species, c_A ~ Beta(2,2) (or centred on mean_cA), c_B = 1 - c_A."""
    rng = np.random.default_rng(seed)
    x = fcc_sites(n, a)
    if sigma > 0:
        x = x + rng.normal(0.0, sigma, size=x.shape)
    L = n * a
    s = _wrap(x / L)
    N = len(s)
    w = rng.uniform(w_lo, w_hi, size=(N, nt))
    alpha = 1.0 / (w * w)
    if nt == 1:
        c = np.ones((N, 1))
    else:
        cA = rng.beta(2.0, 2.0, size=N)
        if mean_cA is not None:
            cA = np.clip(cA + (mean_cA - 0.5), 0.01, 0.99)
        c = np.zeros((N, nt))
        c[:, 0] = cA
        c[:, 1] = 1.0 - cA
        if nt > 2:
            c[:, 1:] = (1.0 - cA)[:, None] / (nt - 1)
    return Config(L, s, [sp.name for sp in ALL_SPECIES[:nt]], [sp.mass for sp in ALL_SPECIES[:nt]],
                  alpha=alpha, c=c)


def make_dmd_cell(nx, ny, nz, a=3.58, sigma=0.0, seed=0, nt=2, w_lo=0.08, w_hi=0.15, mean_cA=None) -> Config:
    """One periodic DMD cell of nx x ny x nz FCC unit cells (box diag(nx, ny, nz) a):
    alpha = 1/w^2 with w ~ U(w_lo, w_hi) A per site and species, c_A ~ Beta(2,2)
    shifted to mean_cA (clipped to [0.01, 0.99]) when given, c_B = 1 - c_A."""
    rng = np.random.default_rng(seed)
    x = fcc_box(nx, ny, nz, a)
    if sigma > 0:
        x = x + rng.normal(0.0, sigma, size=x.shape)
    edges = np.array([nx, ny, nz], dtype=np.float64) * a
    s = _wrap(x / edges)
    N = len(s)
    w = rng.uniform(w_lo, w_hi, size=(N, nt))
    alpha = 1.0 / (w * w)
    if nt == 1:
        c = np.ones((N, 1))
    else:
        cA = rng.beta(2.0, 2.0, size=N)
        if mean_cA is not None:
            cA = np.clip(cA + (mean_cA - 0.5), 0.01, 0.99)
        c = np.zeros((N, nt))
        c[:, 0] = cA
        c[:, 1:] = (1.0 - cA)[:, None] / (nt - 1)
    return Config(float(edges[0]), s, [sp.name for sp in ALL_SPECIES[:nt]], [sp.mass for sp in ALL_SPECIES[:nt]],
                  alpha=alpha, c=c, extra={"H": np.diag(edges)})


def make_batch_cells(ncells=512, seed=2024, lo=500, hi=8000, a=3.58, sigma=0.0, nt=2):
    """Cells of the batched form: site counts log-uniform in [lo, hi], rounded
    to whole FCC unit cells (4 nx ny nz sites), cubic or slab (nx = ny != nz)
    with equal odds; per cell a mean c_A ~ U(0.1, 0.9), per site w ~ U(0.08, 0.15) A."""
    rng = np.random.default_rng(seed)
    cells = []
    for k in range(ncells):
        target = float(np.exp(rng.uniform(np.log(lo), np.log(hi)))) / 4.0
        if rng.uniform() < 0.5:
            n = max(2, int(round(target ** (1.0 / 3.0))))
            shape = (n, n, n)
        else:
            nz = max(2, int(round(target ** (1.0 / 3.0) / 2.0)))
            nxy = max(2, int(round(np.sqrt(target / nz))))
            shape = (nxy, nxy, nz)
        shape = list(shape)
        while 4 * np.prod(shape) > hi:
            shape[int(np.argmax(shape))] -= 1
        while 4 * np.prod(shape) < lo:
            shape[int(np.argmin(shape))] += 1
        cells.append(make_dmd_cell(*shape, a=a, sigma=sigma, seed=int(rng.integers(1 << 31)), nt=nt,
                                   mean_cA=float(rng.uniform(0.1, 0.9))))
    return cells


def write_cfg(path: str, cfg: Config):
    """Extended CFG with .NO_VELOCITY.; DMD lines are s alpha c (read_cfg.cpp:562-627).

    Atoms are grouped by type (a mass line and a name line open each group,
    read_cfg.cpp:589-605); in DMD mode every site is listed under the first
    species and the others are declared with empty groups so that the reader
    registers all of them.
    """
    nt = len(cfg.names)
    with open(path, "w") as fp:
        fp.write("Number of particles = %d\n" % cfg.natms)
        fp.write("A = 1.0 Angstrom (basic length-scale)\n")
        Hm = cfg.H()
        for i in range(3):
            for j in range(3):
                fp.write("H0(%d,%d) = %.17g A\n" % (i + 1, j + 1, Hm[i][j]))
        fp.write(".NO_VELOCITY.\n")
        fp.write("entry_count = %d\n" % (3 + 2 * nt if cfg.dmd else 3))
        if cfg.dmd:
            fp.write("%.17g\n%s\n" % (cfg.masses[0], cfg.names[0]))
            rows = np.concatenate([cfg.s, cfg.alpha, cfg.c], axis=1)
            for row in rows:
                fp.write(" ".join("%.17g" % v for v in row) + "\n")
            for t in range(1, nt):
                fp.write("%.17g\n%s\n" % (cfg.masses[t], cfg.names[t]))
        else:
            for t in range(nt):
                fp.write("%.17g\n%s\n" % (cfg.masses[t], cfg.names[t]))
                for row in cfg.s[cfg.type == t]:
                    fp.write("%.17g %.17g %.17g\n" % tuple(row))


def md_order(cfg: Config) -> np.ndarray:
    """Index permutation the CFG reader applies (atoms grouped by type)."""
    if cfg.dmd:
        return np.arange(cfg.natms)
    return np.concatenate([np.nonzero(cfg.type == t)[0] for t in range(len(cfg.names))])


def write_script(path: str, cfg_path: str, dmd: bool, skin: float = 0.5, extra=()):
    with open(path, "w") as fp:
        fp.write("mode %s\n" % ("dmd" if dmd else "md"))
        fp.write("skin %.17g\n" % skin)
        fp.write("read cfg %s\n" % cfg_path)
        for line in extra:
            fp.write(line + "\n")


def dmd_coef_args(pot_path: str, r_crd=3.0, n_quad=3, alpha_min=20.0, alpha_max=1000.0, T=600.0, fmt="FS"):
    """Arguments of the DMD ``ff_coef`` command (ff_dmd_I.cpp:735-796)."""
    return ["ff_coef", "%.17g" % r_crd, str(n_quad), "%.17g" % alpha_min, "%.17g" % alpha_max,
            "%.17g" % T, fmt, pot_path]


def write_workload(dirpath: str, kind: str, **kw) -> dict:
    """Write a complete workload (cfg + potential + script) and describe it.

    kind: "eam" (FCC EAM crystal, tabulated), "fs" (analytic FS), "dmd" (binary DMD).
    """
    os.makedirs(dirpath, exist_ok=True)
    skin = kw.pop("skin", 0.5)
    box = kw.pop("box", None)  # optional 3x3 lower-triangular H (rows = box vectors); s is kept
    out = {"kind": kind, "dir": dirpath, "skin": skin}
    if kind == "eam":
        nt = kw.pop("nt", 1)
        fmt = kw.pop("fmt", "SetFL")
        cfg = make_md_config(nt=nt, **kw)
        if fmt == "FuncFL":
            # one single-element file per species
            pots = []
            for sp in (SPECIES_A, SPECIES_B)[:nt]:
                pots.append(os.path.join(dirpath, f"pot_{sp.name}.funcfl"))
                write_funcfl(pots[-1], sp)
            pot = pots[0]
            out["coef"] = ["ff_coef", fmt] + pots
        else:
            tables = make_tables((SPECIES_A, SPECIES_B)[:nt])
            pot = os.path.join(dirpath, "pot.eam")
            (write_fs if fmt == "FS" else write_setfl)(pot, tables)
            out["coef"] = ["ff_coef", fmt, pot]
        out["style"] = "EAM"
    elif kind == "fs":
        nt = kw.pop("nt", 1)
        cfg = make_md_config(nt=nt, **kw)
        coeffs = make_fs_coeffs(nt)
        pot = os.path.join(dirpath, "pot.fs_coef")
        write_fs_coeffs(pot, coeffs)
        out["coef"] = ["ff_coef", pot]
        out["style"] = "FS"
    elif kind == "dmd":
        style = kw.pop("style", "DMD_I")
        coef_kw = {k: kw.pop(k) for k in ("r_crd", "n_quad", "alpha_min", "alpha_max", "T") if k in kw}
        cfg = kw.pop("cfg", None) or make_dmd_config(**kw)
        nt = len(cfg.names)
        tables = make_tables(ALL_SPECIES[:nt])
        pot = os.path.join(dirpath, "pot.fs")
        write_fs(pot, tables)
        out["coef"] = dmd_coef_args(pot, **coef_kw)
        out["style"] = style
    else:
        raise ValueError(kind)
    if box is not None:
        cfg.extra["H"] = np.array(box, dtype=np.float64)
    cfg_path = os.path.join(dirpath, "conf.cfg")
    write_cfg(cfg_path, cfg)
    script = os.path.join(dirpath, "in.mapp")
    write_script(script, cfg_path, cfg.dmd, skin)
    out.update(cfg=cfg, cfg_path=cfg_path, script=script, pot=pot)
    return out
