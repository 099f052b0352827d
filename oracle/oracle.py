"""TEST INFRASTRUCTURE ONLY — Python access to the two CPU oracles.

* ``Restatement``: the FP64 C restatement in ``oracle/lbm_oracle.c``
  (built to ``oracle/liblbm_oracle.so``).
* ``Reference``: the reference's own step compiled as host C++ by
  ``oracle/build_ref.sh`` (``oracle/_ref/libref_<lattice>_<variant>.so``).

Only tests, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` use
this module; the product library never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "liblbm_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

COMPAT_D3Q15_MINV_ZERO = 1 << 0
COMPAT_MEQ_INT_DIV = 1 << 1
COMPAT_ZH_Z_UX = 1 << 2
COMPAT_MRTPOR_INPLACE = 1 << 3
COMPAT_AS_IS = (COMPAT_D3Q15_MINV_ZERO | COMPAT_MEQ_INT_DIV | COMPAT_ZH_Z_UX
                | COMPAT_MRTPOR_INPLACE)

LATTICES = {"d2q9": (0, 2, 9), "d3q15": (1, 3, 15)}

_P = ctypes.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def build_restatement(force: bool = False) -> str:
    """Compile oracle/lbm_oracle.c with the system gcc (OpenMP)."""
    src = os.path.join(HERE, "lbm_oracle.c")
    if force or not os.path.exists(RESTATEMENT_SO) or \
            os.path.getmtime(RESTATEMENT_SO) < os.path.getmtime(src):
        subprocess.check_call([
            "/usr/bin/gcc", "-O2", "-fopenmp", "-fPIC", "-shared",
            "-ffp-contract=off", "-fno-fast-math", src, "-lm", "-o", RESTATEMENT_SO])
    return RESTATEMENT_SO


class _OrcConfig(ctypes.Structure):
    _fields_ = [("lattice", ctypes.c_int), ("length", ctypes.c_int * 3),
                ("tau", ctypes.c_double), ("tau_mrt", ctypes.c_double * 15),
                ("c_smag", ctypes.c_double), ("collision_type", ctypes.c_int),
                ("forcing", ctypes.c_int), ("macro_bc", ctypes.c_int),
                ("micro_bc", ctypes.c_int), ("compat", ctypes.c_uint)]


@dataclass
class Case:
    """One time-step problem in the reference's terms (ixd node order).

    Arrays: geometry (N), force (DIM,N), macro/micro (N int32), u (DIM,N),
    rho (N), f0 (Q,N natural layout) — any may be None.
    """
    lattice: str
    length: tuple
    tau: float = 0.8
    tau_mrt: tuple = ()
    c_smag: float = 0.0
    collision_type: int = 0
    forcing: bool = False
    macro_bc: bool = False
    micro_bc: bool = False
    compat: int = 0
    geometry: np.ndarray | None = None
    force: np.ndarray | None = None
    macro: np.ndarray | None = None
    micro: np.ndarray | None = None
    u: np.ndarray | None = None
    rho: np.ndarray | None = None
    f0: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def dim(self):
        return LATTICES[self.lattice][1]

    @property
    def q(self):
        return LATTICES[self.lattice][2]

    @property
    def n(self):
        return int(np.prod(self.length[:self.dim]))

    def arrays(self):
        """Contiguous float64/int32 copies (None kept) in the oracle layouts."""
        def f64(a, shape):
            return None if a is None else np.ascontiguousarray(a, np.float64).reshape(shape)

        def i32(a):
            return None if a is None else np.ascontiguousarray(a, np.int32).reshape(self.n)
        d, q, n = self.dim, self.q, self.n
        return dict(geometry=f64(self.geometry, n), force=f64(self.force, (d, n)),
                    macro=i32(self.macro), micro=i32(self.micro), u=f64(self.u, (d, n)),
                    rho=f64(self.rho, n), f0=f64(self.f0, (q, n)))


class Restatement:
    """FP64 restatement; natural layout, two buffers."""

    def __init__(self, case: Case):
        lib = ctypes.CDLL(build_restatement())
        lib.orc_create.restype = _P
        lib.orc_create.argtypes = [ctypes.POINTER(_OrcConfig)] + [_P] * 7
        for name in ("orc_run",):
            getattr(lib, name).argtypes = [_P, ctypes.c_int, ctypes.c_int]
        lib.orc_get_f.argtypes = [_P, _P]
        lib.orc_get_macros.argtypes = [_P, _P, _P]
        lib.orc_destroy.argtypes = [_P]
        lib.orc_tables.argtypes = [_P] * 6
        lib.orc_equilibrium_field.argtypes = [_P] * 4
        lib.orc_set_tau_field.argtypes = [_P, _P]
        self.lib, self.case = lib, case
        cfg = _OrcConfig()
        cfg.lattice = LATTICES[case.lattice][0]
        for d in range(3):
            cfg.length[d] = case.length[d] if d < len(case.length) else 1
        cfg.tau = case.tau
        for i, v in enumerate(case.tau_mrt):
            cfg.tau_mrt[i] = v
        cfg.c_smag = case.c_smag
        cfg.collision_type = case.collision_type
        cfg.forcing = int(case.forcing)
        cfg.macro_bc = int(case.macro_bc)
        cfg.micro_bc = int(case.micro_bc)
        cfg.compat = case.compat
        self._keep = a = case.arrays()
        self.h = lib.orc_create(ctypes.byref(cfg), _ptr(a["geometry"]), _ptr(a["force"]),
                                _ptr(a["macro"]), _ptr(a["micro"]), _ptr(a["u"]),
                                _ptr(a["rho"]), _ptr(a["f0"]))

    def run(self, nsteps: int, store_last: bool = True):
        self.lib.orc_run(self.h, nsteps, int(store_last))

    def f(self):
        out = np.empty((self.case.q, self.case.n))
        self.lib.orc_get_f(self.h, _ptr(out))
        return out

    def macros(self):
        rho = np.empty(self.case.n)
        u = np.empty((self.case.dim, self.case.n))
        self.lib.orc_get_macros(self.h, _ptr(rho), _ptr(u))
        return rho, u

    def tables(self):
        q, d = self.case.q, self.case.dim
        e = np.zeros((d, q), np.int32)
        w, opp = np.zeros(q), np.zeros(q, np.int32)
        M, Minv = np.zeros((q, q)), np.zeros((q, q))
        self.lib.orc_tables(self.h, _ptr(e), _ptr(w), _ptr(opp), _ptr(M), _ptr(Minv))
        return e, w, opp, M, Minv

    def equilibrium(self, rho, u):
        out = np.empty((self.case.q, self.case.n))
        rho = np.ascontiguousarray(rho, np.float64)
        u = np.ascontiguousarray(u, np.float64)
        self.lib.orc_equilibrium_field(self.h, _ptr(rho), _ptr(u), _ptr(out))
        return out

    def set_tau_field(self, tau):
        """Per-node relaxation times (N) for the following steps, or None."""
        self._tau = None if tau is None else np.ascontiguousarray(tau, np.float64)
        self.lib.orc_set_tau_field(self.h, _ptr(self._tau))

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reference_available(lattice: str, variant: str = "asis") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{lattice}_{variant}.so"))


class Reference:
    """The reference's own step, host-compiled (oracle/_ref)."""

    _libs: dict = {}

    def __init__(self, case: Case, variant: str = "asis", nthreads: int = 0):
        path = os.path.join(REF_DIR, f"libref_{case.lattice}_{variant}.so")
        if path not in Reference._libs:
            lib = ctypes.CDLL(path)
            lib.ref_create.restype = _P
            lib.ref_create.argtypes = [_P, ctypes.c_double, _P, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int] + [_P] * 7
            lib.ref_run.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            lib.ref_get_f.argtypes = [_P, ctypes.c_int, _P]
            lib.ref_get_macros.argtypes = [_P, _P, _P]
            lib.ref_destroy.argtypes = [_P]
            lib.ref_tables.argtypes = [_P] * 5
            Reference._libs[path] = lib
        self.lib = lib = Reference._libs[path]
        self.case, self.t, self.nthreads = case, 0, nthreads
        length = np.array(list(case.length) + [1] * (3 - len(case.length)), np.int32)
        tau_mrt = np.zeros(15)
        tau_mrt[:len(case.tau_mrt)] = case.tau_mrt
        self._keep = a = case.arrays()
        self._keep2 = (length, tau_mrt)
        self.h = lib.ref_create(_ptr(length), case.tau, _ptr(tau_mrt), case.c_smag,
                                case.collision_type, int(case.forcing), int(case.macro_bc),
                                int(case.micro_bc), _ptr(a["geometry"]), _ptr(a["force"]),
                                _ptr(a["macro"]), _ptr(a["micro"]), _ptr(a["u"]),
                                _ptr(a["rho"]), _ptr(a["f0"]))

    def run(self, nsteps: int, store_last: bool = True):
        self.lib.ref_run(self.h, self.t, nsteps, int(store_last), self.nthreads)
        self.t += nsteps

    def f(self):
        out = np.empty((self.case.q, self.case.n))
        self.lib.ref_get_f(self.h, self.t, _ptr(out))
        return out

    def macros(self):
        rho = np.empty(self.case.n)
        u = np.empty((self.case.dim, self.case.n))
        self.lib.ref_get_macros(self.h, _ptr(rho), _ptr(u))
        return rho, u

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
