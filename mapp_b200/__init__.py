"""mapp_b200: B200-native force-field hot path of MAPP (neighbour list,
EAM / Finnis-Sinclair / DMD energies, forces and chemical potentials).

The compute path is the CUDA library ``libmapp_b200.so`` (C ABI declared in
``include/mapp_b200.h``).  This module is a thin ctypes mirror of that ABI,
shaped like the reference's own objects: a :class:`System` holds one MAPP
system (Atoms + Neighbor + ForceField) and exposes the ForceField virtuals
(``coef``, ``init``, ``force_calc``, ``energy_calc``, ``create_2nd_neigh_lst``,
``c_d_calc``, ``calc_g``) and the Atoms updates the reference's callers use
(``update_0`` via :meth:`System.update_x`, ``update(c)`` via
:meth:`System.update_c`).  There is no CPU path: without the library or a GPU
every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmapp_b200.so")

MG_FORM_FP64, MG_FORM_FP32, MG_FORM_MLP = 0, 1, 2
MG_MIN_LBFGS, MG_MIN_CG = 0, 1
MG_LAUNCH_WHOLE_GPU = -1
MG_ERR_TIMEOUT = 8
MG_MLP_ACT_POLY = 0
MG_MLP_ACT_TANH = 1
MG_MLP_ACT_SPLIT = 2
ERRORS = {1: "ARG", 2: "FILE", 3: "FORMAT", 4: "STATE", 5: "CUDA", 6: "CAPACITY", 7: "UNSUPPORTED", 8: "TIMEOUT", 9: "DOMAIN"}

# Every exported entry point of include/mapp_b200.h with its ctypes signature.
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
SIGNATURES = {
    "mg_last_error": (C.c_char_p, []),
    "mg_version": (C.c_int, []),
    "mg_create": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mg_destroy": (C.c_int, [_P]),
    "mg_set_stream": (C.c_int, [_P, _P]),
    "mg_set_form": (C.c_int, [_P, C.c_int]),
    "mg_atoms_set_types": (C.c_int, [_P, C.c_int, C.POINTER(C.c_char_p), _D]),
    "mg_atoms_set_box": (C.c_int, [_P, _P]),
    "mg_atoms_set_skin": (C.c_int, [_P, C.c_double]),
    "mg_atoms_set": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "mg_atoms_update_x": (C.c_int, [_P, _P, _I]),
    "mg_atoms_update_c": (C.c_int, [_P, _P]),
    "mg_atoms_get_x": (C.c_int, [_P, _P]),
    "mg_atoms_get_ghosts": (C.c_int, [_P, _P, _P]),
    "mg_ff_coef": (C.c_int, [_P, C.c_int, C.POINTER(C.c_char_p)]),
    "mg_ff_init": (C.c_int, [_P]),
    "mg_ff_force_calc": (C.c_int, [_P, C.c_int, _P, _D]),
    "mg_ff_energy_calc": (C.c_int, [_P, _D]),
    "mg_ff_create_2nd_neigh_lst": (C.c_int, [_P]),
    "mg_ff_c_d_calc": (C.c_int, [_P, _P]),
    "mg_ff_calc_g": (C.c_int, [_P, C.c_int, C.c_double, _P, _P, _D]),
    "mg_ff_fin": (C.c_int, [_P]),
    "mg_neighbor_create_list": (C.c_int, [_P]),
    "mg_neighbor_counts": (C.c_int, [_P, _I, _I, C.POINTER(C.c_longlong)]),
    "mg_neighbor_get_list": (C.c_int, [_P, _P, _P]),
    "mg_get_vector": (C.c_int, [_P, C.c_char_p, _P]),
    "mg_get_int_vector": (C.c_int, [_P, C.c_char_p, _P]),
    "mg_last_time": (C.c_int, [_P, C.c_char_p, _D]),
    "mg_set_timing": (C.c_int, [_P, C.c_int]),
    "mg_fs_energy_noalloc": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P]),
    "mg_mlp_nparam": (C.c_int, []),
    "mg_mlp_init": (C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_ulonglong]),
    "mg_mlp_train": (C.c_int, [_P, C.c_longlong, C.c_int, C.c_int, C.c_double, C.c_ulonglong, _D]),
    "mg_mlp_loss_history": (C.c_int, [_P, C.c_int, _P]),
    "mg_mlp_state": (C.c_int, [_P, _P, _P, _P, _P]),
    "mg_mlp_eval": (C.c_int, [_P, C.c_int, _P, _P]),
    "mg_mlp_grad": (C.c_int, [_P, C.c_int, _P, _P, _P, _D]),
    "mg_mlp_audit": (C.c_int, [_P, _D, C.POINTER(C.c_longlong)]),
    "mg_batch_create": (C.c_int, [_P, C.POINTER(C.c_void_p)]),
    "mg_batch_destroy": (C.c_int, [_P]),
    "mg_batch_add_cell": (C.c_int, [_P, C.c_int, _P, _P, _P, _I]),
    "mg_batch_set_params": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
    "mg_batch_set_form": (C.c_int, [_P, C.c_int]),
    "mg_batch_set_tuning": (C.c_int, [_P, C.c_int, C.c_char_p]),
    "mg_batch_set_launch": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    "mg_batch_set_limits": (C.c_int, [_P, C.c_longlong, C.c_double]),
    "mg_mlp_set_activation": (C.c_int, [_P, C.c_int]),
    "mg_batch_relax": (C.c_int, [_P, _P]),
    "mg_batch_cell_result": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "mg_min_lbfgs": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _P, _P]),
    "mg_min_cg": (C.c_int, [_P, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _P, _P]),
    "mg_batch_set_method": (C.c_int, [_P, C.c_int]),
    "mg_clock_adams": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, _P, C.POINTER(C.c_longlong)]),
    "mg_bdf_defaults": (None, [_P]),
    "mg_clock_bdf": (C.c_int, [_P, C.c_int, _P, _P, _I, C.POINTER(C.c_longlong)]),
    "mg_md_nh": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _P,
                           C.c_int, _P, _P, _I]),
    "mg_cfg_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "mg_cfg_info": (C.c_int, [_P, _I, _I, _P, _I]),
    "mg_cfg_types": (C.c_int, [_P, _P, C.c_int, _P]),
    "mg_cfg_atoms": (C.c_int, [_P, _P, _P, _P, _P]),
    "mg_cfg_free": (C.c_int, [_P]),
    "mg_cfg_write_arrays": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int, _P, _P,
                                      _P, _P, _P]),
    "mg_cfg_write": (C.c_int, [_P, C.c_char_p, C.c_int]),
}


class BatchStats(C.Structure):
    """mg_batch_stats (include/mapp_b200.h)."""

    _fields_ = [("relax_ms", C.c_double), ("build_ms", C.c_double), ("tune_ms", C.c_double),
                ("iterations", C.c_longlong), ("evaluations", C.c_longlong), ("rebuild_rounds", C.c_int),
                ("converged", C.c_int), ("bps1", C.c_int), ("bps2", C.c_int), ("lbfgs_threads", C.c_int),
                ("from_cache", C.c_int), ("lbfgs_cluster", C.c_int)]


class CellResult(C.Structure):
    """mg_cell_result (include/mapp_b200.h)."""

    _fields_ = [("energy", C.c_double), ("max_f", C.c_double), ("t_ms", C.c_double), ("code", C.c_int),
                ("iterations", C.c_int), ("evaluations", C.c_int), ("natms", C.c_int)]


class FsCoeffs(C.Structure):
    """mg_fs_coeffs of include/mapp_b200.h (analytic Finnis-Sinclair coefficients)."""

    _fields_ = [("ntypes", C.c_int), ("chk", C.c_int * 10), ("A", C.c_double * 4),
                ("t1", (C.c_double * 4) * 4), ("t2", (C.c_double * 4) * 4),
                ("cut_rho", C.c_double * 10), ("cut_phi", C.c_double * 10),
                ("k1", C.c_double * 10), ("k2", C.c_double * 10), ("k3", C.c_double * 10)]


class BdfOpts(C.Structure):
    """mg_bdf_opts: the options of "clock bdf" (clock_bdf.cpp:14-111)."""
    _fields_ = [("max_order", C.c_int), ("max_iter", C.c_int), ("min_gamma", C.c_double),
                ("gamma_red", C.c_double), ("slope", C.c_double), ("m_tol", C.c_double), ("a_tol", C.c_double),
                ("e_tol", C.c_double), ("min_del_t", C.c_double), ("max_del_t", C.c_double),
                ("initial_del_t", C.c_double)]


class MGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mapp_b200 error {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"mapp_b200 CUDA library not built ({path}); run python -m mapp_b200.build")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    """Pointer of a numpy array, a torch tensor (host or device) or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(type(a))


def _check(rc):
    if rc != 0:
        raise MGError(rc, load_library().mg_last_error().decode())


class System:
    """One MAPP system on one GPU, driven through the C ABI."""

    def __init__(self, style: str, device: int = 0):
        L = load_library()
        h = C.c_void_p()
        _check(L.mg_create(style.encode(), device, C.byref(h)))
        self.h = h
        self.style = style
        self.dmd = style.startswith("DMD")
        self.nt = 0
        self.natms = 0

    def close(self):
        if getattr(self, "h", None):
            load_library().mg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def x_dim(self):
        return 3 + self.nt if self.dmd else 3

    # ---- setup -----------------------------------------------------------
    def set_types(self, names, masses):
        self.nt = len(names)
        arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
        m = np.ascontiguousarray(masses, dtype=np.float64)
        _check(load_library().mg_atoms_set_types(self.h, len(names), arr, m.ctypes.data_as(_D)))

    def set_box(self, H):
        H = np.ascontiguousarray(H, dtype=np.float64).reshape(9)
        _check(load_library().mg_atoms_set_box(self.h, H.ctypes.data))

    def set_skin(self, skin):
        _check(load_library().mg_atoms_set_skin(self.h, float(skin)))

    def set_atoms(self, x_frac, type=None, c=None):
        x = np.ascontiguousarray(x_frac, dtype=np.float64)
        self.natms = x.shape[0]
        t = None if type is None else np.ascontiguousarray(type, dtype=np.int32)
        cc = None if c is None else np.ascontiguousarray(c, dtype=np.float64)
        _check(load_library().mg_atoms_set(self.h, self.natms, _ptr(x), _ptr(t), _ptr(cc)))

    def set_stream(self, stream_ptr: int):
        _check(load_library().mg_set_stream(self.h, stream_ptr))

    def set_form(self, form: int):
        _check(load_library().mg_set_form(self.h, form))

    def coef(self, args):
        arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
        _check(load_library().mg_ff_coef(self.h, len(args), arr))

    def init(self):
        _check(load_library().mg_ff_init(self.h))

    # ---- ForceField ------------------------------------------------------
    def force_calc(self, st_clc=1, f=None):
        """Returns (f, en_st); f may be a preallocated host/device buffer."""
        out = f if f is not None else np.zeros((self.natms, self.x_dim))
        en = np.zeros(7)
        _check(load_library().mg_ff_force_calc(self.h, st_clc, _ptr(out), en.ctypes.data_as(_D)))
        return out, (en if st_clc else en[:1])

    def energy_calc(self):
        e = C.c_double(0.0)
        _check(load_library().mg_ff_energy_calc(self.h, C.byref(e)))
        return e.value

    def create_2nd_neigh_lst(self):
        _check(load_library().mg_ff_create_2nd_neigh_lst(self.h))

    def c_d_calc(self, out=None):
        o = out if out is not None else np.zeros((self.natms, self.nt))
        _check(load_library().mg_ff_c_d_calc(self.h, _ptr(o)))
        return o

    def calc_g(self, a, alpha, chk=0, g=None):
        aa = a if not isinstance(a, np.ndarray) else np.ascontiguousarray(a, dtype=np.float64)
        gg = g if g is not None else np.zeros((self.natms, self.nt))
        cost = C.c_double(0.0)
        _check(load_library().mg_ff_calc_g(self.h, chk, float(alpha), _ptr(aa), _ptr(gg), C.byref(cost)))
        return cost.value, gg

    def fin(self):
        _check(load_library().mg_ff_fin(self.h))

    # ---- Atoms -----------------------------------------------------------
    def update_x(self, x, report=True):
        """Atoms::update_0 with new positions. With report the call waits for
        the skin test and returns whether the list was rebuilt; without, the
        test is settled by the next call that needs the list (force_calc reads
        it with its results) and None is returned."""
        xx = x if not isinstance(x, np.ndarray) else np.ascontiguousarray(x, dtype=np.float64)
        if not report:
            _check(load_library().mg_atoms_update_x(self.h, _ptr(xx), None))
            return None
        r = C.c_int(0)
        _check(load_library().mg_atoms_update_x(self.h, _ptr(xx), C.byref(r)))
        return r.value

    def update_c(self, c):
        cc = c if not isinstance(c, np.ndarray) else np.ascontiguousarray(c, dtype=np.float64)
        _check(load_library().mg_atoms_update_c(self.h, _ptr(cc)))

    def get_x(self):
        x = np.zeros((self.natms, self.x_dim))
        _check(load_library().mg_atoms_get_x(self.h, x.ctypes.data))
        return x

    def counts(self):
        n, g, p = C.c_int(0), C.c_int(0), C.c_longlong(0)
        _check(load_library().mg_neighbor_counts(self.h, C.byref(n), C.byref(g), C.byref(p)))
        return dict(natms=n.value, nph=g.value, npairs=p.value)

    def ghosts(self):
        c = self.counts()
        x = np.zeros((c["nph"], self.x_dim))
        o = np.zeros(c["nph"], dtype=np.int32)
        _check(load_library().mg_atoms_get_ghosts(self.h, x.ctypes.data, o.ctypes.data))
        return x, o

    def neighbor_list(self):
        c = self.counts()
        sizes = np.zeros(self.natms, dtype=np.int32)
        pairs = np.zeros(max(c["npairs"], 1), dtype=np.int32)
        _check(load_library().mg_neighbor_get_list(self.h, sizes.ctypes.data, pairs.ctypes.data))
        return sizes, pairs[:c["npairs"]]

    def rebuild_list(self):
        _check(load_library().mg_neighbor_create_list(self.h))

    def vector(self, name):
        n = self.natms * (1 if name == "rho" else self.nt)
        out = np.zeros(n)
        _check(load_library().mg_get_vector(self.h, name.encode(), out.ctypes.data))
        return out

    def crd(self):
        c = self.counts()
        out = np.zeros(c["natms"] + c["nph"], dtype=np.int32)
        _check(load_library().mg_get_int_vector(self.h, b"crd", out.ctypes.data))
        return out

    # ---- learned form ------------------------------------------------------
    def mlp_set_activation(self, act):
        _check(load_library().mg_mlp_set_activation(self.h, act))

    def mlp_init(self, r_lo=1.8, r_hi=5.0, w_lo=0.05, w_hi=0.20, seed=1):
        _check(load_library().mg_mlp_init(self.h, r_lo, r_hi, w_lo, w_hi, seed))

    def mlp_train(self, nsamples=2_000_000, steps=20_000, batch=4096, lr=1e-3, seed=7):
        loss = C.c_double(0.0)
        _check(load_library().mg_mlp_train(self.h, nsamples, steps, batch, lr, seed, C.byref(loss)))
        return loss.value

    def mlp_loss_history(self, n):
        out = np.zeros(n, dtype=np.float32)
        _check(load_library().mg_mlp_loss_history(self.h, n, out.ctypes.data))
        return out

    def mlp_state(self, params=None, scaling=None):
        L = load_library()
        npar = L.mg_mlp_nparam()
        pout = np.zeros(npar, dtype=np.float32)
        sout = np.zeros(12, dtype=np.float32)
        pin = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        sin = None if scaling is None else np.ascontiguousarray(scaling, dtype=np.float32)
        _check(L.mg_mlp_state(self.h, pout.ctypes.data, _ptr(pin), sout.ctypes.data, _ptr(sin)))
        return pout, sout

    def mlp_eval(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], 6), dtype=np.float32)
        _check(load_library().mg_mlp_eval(self.h, x.shape[0], x.ctypes.data, y.ctypes.data))
        return y

    def mlp_grad(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(load_library().mg_mlp_nparam(), dtype=np.float32)
        loss = C.c_double(0.0)
        _check(load_library().mg_mlp_grad(self.h, x.shape[0], x.ctypes.data, y.ctypes.data, g.ctypes.data,
                                          C.byref(loss)))
        return g, loss.value

    def mlp_audit(self):
        err = np.zeros(6)
        cnt = np.zeros(2, dtype=np.int64)
        _check(load_library().mg_mlp_audit(self.h, err.ctypes.data_as(_D), cnt.ctypes.data_as(C.POINTER(C.c_longlong))))
        return err, cnt

    def min_lbfgs(self, m=5, max_iter=10000, fmax_tol=1e-5, energy_tol=1e-8, max_halvings=60, cluster=0):
        """Device-resident L-BFGS relaxation of this system (mg_min_lbfgs);
        returns (result, stats) dicts.  cluster: CTAs per L-BFGS step, 0 = autotune."""
        r = CellResult()
        st = BatchStats()
        _check(load_library().mg_min_lbfgs(self.h, m, max_iter, fmax_tol, energy_tol, max_halvings, cluster,
                                           C.byref(r), C.byref(st)))
        return ({k: getattr(r, k) for k, _ in CellResult._fields_}, {k: getattr(st, k) for k, _ in BatchStats._fields_})

    def clock_adams(self, order, steps, dt):
        """Adams clock of this DMD system on the device (mg_clock_adams).
        Returns dict(c, err, n_calc_g)."""
        err = np.zeros(max(steps, 1))
        ncg = C.c_longlong(0)
        _check(load_library().mg_clock_adams(self.h, order, steps, dt, err.ctypes.data, C.byref(ncg)))
        return {"c": self.vector("c"), "err": err[:steps], "n_calc_g": int(ncg.value)}

    def clock_bdf(self, steps, **opts):
        """BDF clock of this DMD system on the device (mg_clock_bdf); options
        as the fields of BdfOpts (unset ones keep the reference's defaults).
        Returns dict(c, n_calc_g, steps, del_t, order, t): per step its size,
        the order it ran at and the time after it; t is the final time."""
        lib = load_library()
        o = BdfOpts()
        lib.mg_bdf_defaults(C.byref(o))
        names = {k for k, _ in BdfOpts._fields_}
        for k, v in opts.items():
            if k not in names:
                raise ValueError(f"unknown clock bdf option {k}")
            setattr(o, k, v)
        hist = np.zeros(3 * max(steps, 1))
        ncg = C.c_longlong(0)
        taken = C.c_int(0)
        _check(lib.mg_clock_bdf(self.h, steps, C.byref(o), hist.ctypes.data, C.byref(taken), C.byref(ncg)))
        k = taken.value
        h = hist[: 3 * k].reshape(-1, 3)
        return {"c": self.vector("c"), "n_calc_g": int(ncg.value), "steps": k, "del_t": h[:, 0],
                "order": h[:, 1].astype(int), "t": float(h[-1, 2]) if k else 0.0}

    def md_nh(self, t_tar, t_period, steps, dt, boltz, xd=None, seed=0, eta_iteration=1, eta_chains=3):
        """Nose-Hoover NVT run of this EAM / FS system on the device (mg_md_nh).
        xd: initial velocities [natms][3] (rescaled to t_tar), or seed > 0 for
        create_vel.  Returns dict(x, xd, energy, virial, ke, t, eta_d, rebuilds)."""
        n = self.natms
        xin = None
        if seed <= 0:
            xin = np.ascontiguousarray(np.asarray(xd, dtype=np.float64).reshape(n, 3))
        vout = np.zeros((n, 3))
        th = np.zeros(9 + eta_chains)
        nreb = C.c_int(0)
        _check(load_library().mg_md_nh(self.h, t_tar, t_period, eta_iteration, eta_chains, dt, boltz, seed,
                                       None if xin is None else xin.ctypes.data, steps, vout.ctypes.data,
                                       th.ctypes.data, C.byref(nreb)))
        return {"x": self.get_x(), "xd": vout, "energy": th[0], "virial": th[1:7], "ke": th[7], "t": th[8],
                "eta_d": th[9:9 + eta_chains], "rebuilds": nreb.value}

    def write_cfg(self, prefix, step=0):
        """WriteCFG's file of this system's current state (mg_cfg_write)."""
        _check(load_library().mg_cfg_write(self.h, str(prefix).encode(), step))
        return "%s.%08d.cfg" % (prefix, step)

    def min_cg(self, max_iter=10000, fmax_tol=1e-5, energy_tol=1e-8, max_halvings=60, cluster=0):
        """Device-resident conjugate-gradient relaxation of this system (mg_min_cg);
        returns (result, stats) dicts like min_lbfgs."""
        r = CellResult()
        st = BatchStats()
        _check(load_library().mg_min_cg(self.h, max_iter, fmax_tol, energy_tol, max_halvings, cluster, C.byref(r),
                                        C.byref(st)))
        return ({k: getattr(r, k) for k, _ in CellResult._fields_}, {k: getattr(st, k) for k, _ in BatchStats._fields_})

    def last_time(self, phase):
        ms = C.c_double(0.0)
        _check(load_library().mg_last_time(self.h, phase.encode(), C.byref(ms)))
        return ms.value

    def set_timing(self, level):
        """Device timing level: 0 none, 1 (default) whole calls, 2 also the
        DMD force call's kernels (last_time("force.*")); each event costs a
        call a few microseconds."""
        _check(load_library().mg_set_timing(self.h, int(level)))


def fs_energy_noalloc(coeffs: "FsCoeffs", natms: int, nall: int, x, type, nbr_off, nbr, energy, stream: int = 0):
    """ForceField_fs::energy_calc from caller-owned device buffers without any
    allocation in the library (mg_fs_energy_noalloc).  x, type, nbr_off and
    nbr must be device tensors; energy may be a host numpy array or a device
    tensor of one double."""
    _check(load_library().mg_fs_energy_noalloc(C.byref(coeffs), natms, nall, _ptr(x), _ptr(type), _ptr(nbr_off),
                                               _ptr(nbr), _ptr(energy), stream))


class Batch:
    """Batched form: independent DMD cells relaxed by L-BFGS together on one GPU
    (mg_batch_*).  `builder` is a DMD System with types, skin and ff_coef set;
    its atoms are replaced while the batch builds each cell's lists."""

    def __init__(self, builder: "System"):
        L = load_library()
        self.builder = builder
        self.nt = builder.nt
        h = C.c_void_p()
        _check(L.mg_batch_create(builder.h, C.byref(h)))
        self.h = h.value
        self.natms = []

    def close(self):
        if getattr(self, "h", None):
            load_library().mg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_cell(self, cfg) -> int:
        """Add a fixtures.Config cell (its box, s + alpha, c)."""
        H = np.ascontiguousarray(cfg.H(), dtype=np.float64)
        x = np.ascontiguousarray(cfg.x_dmd(), dtype=np.float64)
        c = np.ascontiguousarray(cfg.c, dtype=np.float64)
        idx = C.c_int(-1)
        _check(load_library().mg_batch_add_cell(self.h, cfg.natms, H.ctypes.data, x.ctypes.data, c.ctypes.data,
                                                C.byref(idx)))
        self.natms.append(cfg.natms)
        return idx.value

    def set_params(self, m=5, max_iter=10000, fmax_tol=1e-5, energy_tol=1e-8, max_halvings=60):
        _check(load_library().mg_batch_set_params(self.h, m, max_iter, fmax_tol, energy_tol, max_halvings))

    def set_form(self, form):
        _check(load_library().mg_batch_set_form(self.h, form))

    def set_method(self, method):
        """MG_MIN_LBFGS (default) or MG_MIN_CG."""
        _check(load_library().mg_batch_set_method(self.h, method))

    def set_tuning(self, autotune=True, cache_path=None):
        _check(load_library().mg_batch_set_tuning(self.h, int(autotune),
                                                  None if cache_path is None else str(cache_path).encode()))

    def set_launch(self, bps1=0, bps2=0, lbfgs_threads=256, lbfgs_cluster=1):
        _check(load_library().mg_batch_set_launch(self.h, bps1, bps2, lbfgs_threads, lbfgs_cluster))

    def set_limits(self, iteration_budget=0, barrier_wait_s=2.0):
        """Iteration budget of one launch (0: automatic) and grid-barrier wait
        limit; running out of either raises MGError (MG_ERR_TIMEOUT)."""
        _check(load_library().mg_batch_set_limits(self.h, int(iteration_budget), float(barrier_wait_s)))

    def relax(self) -> dict:
        st = BatchStats()
        _check(load_library().mg_batch_relax(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in BatchStats._fields_}

    def cell_result(self, cell: int):
        """(x, f, info): final Cartesian x + alpha and forces (natms x (3 + nt)), result fields."""
        n = self.natms[cell]
        xd = 3 + self.nt
        x = np.zeros((n, xd))
        f = np.zeros((n, xd))
        r = CellResult()
        _check(load_library().mg_batch_cell_result(self.h, cell, x.ctypes.data, f.ctypes.data, C.byref(r)))
        return x, f, {k: getattr(r, k) for k, _ in CellResult._fields_}


def read_cfg(path: str, dmd: bool = False) -> dict:
    """A CFG file as the reference reads it (mg_cfg_*): dict(names, masses, H
    (lower triangular), s (natms x 3, wrapped), and type + v (MD) or alpha + c
    (DMD))."""
    L = load_library()
    h = C.c_void_p()
    _check(L.mg_cfg_read(str(path).encode(), int(dmd), C.byref(h)))
    try:
        n, nty, hv = C.c_int(), C.c_int(), C.c_int()
        H = np.zeros(9)
        _check(L.mg_cfg_info(h, C.byref(n), C.byref(nty), H.ctypes.data, C.byref(hv)))
        names = C.create_string_buffer(64 * max(nty.value, 1))
        masses = np.zeros(max(nty.value, 1))
        _check(L.mg_cfg_types(h, names, 64, masses.ctypes.data))
        N = n.value
        out = {"names": [names.raw[64 * k:64 * (k + 1)].split(b"\0")[0].decode() for k in range(nty.value)],
               "masses": masses[: nty.value].tolist(), "H": H.reshape(3, 3), "has_velocity": bool(hv.value)}
        if dmd:
            nt = nty.value
            x = np.zeros((N, 3 + nt))
            c = np.zeros((N, nt))
            _check(L.mg_cfg_atoms(h, x.ctypes.data, None, c.ctypes.data, None))
            out.update(s=x[:, :3].copy(), alpha=x[:, 3:].copy(), c=c)
        else:
            x = np.zeros((N, 3))
            t = np.zeros(N, dtype=np.int32)
            v = np.zeros((N, 3))
            _check(L.mg_cfg_atoms(h, x.ctypes.data, t.ctypes.data, None, v.ctypes.data))
            out.update(s=x, type=t, v=v)
        return out
    finally:
        L.mg_cfg_free(h)


def write_cfg(prefix: str, step: int, names, masses, H, x, type=None, c=None):
    """WriteCFG's file for host arrays (mg_cfg_write_arrays): x is Cartesian,
    natms x 3 (MD, with type) or natms x (3 + nt) with the alphas (DMD, with c).
    Returns the path of the .cfg file written."""
    L = load_library()
    dmd = c is not None
    nt = len(names)
    name_len = max(len(n) for n in names) + 1
    nb = b"".join(n.encode().ljust(name_len, b"\0") for n in names)
    m = np.ascontiguousarray(masses, dtype=np.float64)
    Hm = np.ascontiguousarray(np.asarray(H, dtype=np.float64).reshape(9))
    xa = np.ascontiguousarray(x, dtype=np.float64)
    ta = None if dmd else np.ascontiguousarray(type, dtype=np.int32)
    ca = np.ascontiguousarray(c, dtype=np.float64) if dmd else None
    _check(L.mg_cfg_write_arrays(str(prefix).encode(), step, int(dmd), xa.shape[0], nt, nb, name_len, m.ctypes.data,
                                 Hm.ctypes.data, xa.ctypes.data, None if dmd else ta.ctypes.data,
                                 ca.ctypes.data if dmd else None))
    return "%s.%08d.cfg" % (prefix, step)


def system_from_workload(w: dict, device: int = 0, skin: float = 0.5) -> System:
    """Build and init a System from a workload written by mapp_b200.fixtures."""
    from .fixtures import md_order

    cfg = w["cfg"]
    s = System(w["style"], device)
    s.set_types(cfg.names, cfg.masses)
    s.set_box(cfg.H())
    s.set_skin(skin)
    if cfg.dmd:
        s.set_atoms(cfg.x_dmd(), c=cfg.c)
    else:
        order = md_order(cfg)
        s.set_atoms(cfg.s[order], type=cfg.type[order])
    s.coef(w["coef"])
    s.init()
    return s
