"""ctypes binding of the lbmc C ABI (include/lbmc.h).

This is the Python mirror of the engine's drop-in boundary: ``Engine`` wraps
``lbmc_init`` / ``lbmc_iterate`` / ``lbmc_fetch`` / ``lbmc_destroy`` exactly,
with the same argument meaning and status codes (errors raise ``LbmcError``
carrying the status and ``lbmc_last_error()``).  It loads the in-tree
``liblbmc.so`` built by ``make -C lbm-c_b200`` and fails loudly when that
library is absent: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbmc.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "lbmc.h")

# enums / flags of include/lbmc.h
OK, ERR_INVALID_ARG, ERR_UNSUPPORTED, ERR_CUDA, ERR_ALLOC, ERR_NAN, ERR_TIMEOUT, ERR_IO, \
    ERR_BUFFER_SIZE, ERR_NO_DEVICE = range(10)
D2Q9, D3Q15 = 0, 1
F32, F16, BF16, F64, F16_SR = 0, 1, 2, 3, 4
BGK, NTPOR, MRT, MRTPOR = 0, 1, 2, 3
INIT_STATIC, INIT_EQUILIBRIUM, INIT_F = 0, 1, 2
STREAM_SHIFT, STREAM_AA = 0, 1
KERNEL_AUTO, KERNEL_DIRECT, KERNEL_PIPELINED = 0, 1, 2
COMPAT_D3Q15_MINV_ZERO = 1 << 0
COMPAT_MEQ_INT_DIV = 1 << 1
COMPAT_ZH_Z_UX = 1 << 2
COMPAT_MRTPOR_INPLACE = 1 << 3
COMPAT_REFERENCE_AS_IS = 0xF
STORE_MACROS, REDUCE_DIAG, SYNC = 1, 2, 4
FIELD_RHO, FIELD_U_X, FIELD_U_Y, FIELD_U_Z, FIELD_F, FIELD_DIAG = range(6)

LATTICE_IDS = {"d2q9": D2Q9, "d3q15": D3Q15}
STORAGE_IDS = {"f32": F32, "f16": F16, "bf16": BF16, "f64": F64, "f16sr": F16_SR}

_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


class Config(ctypes.Structure):
    _fields_ = [("lattice", ctypes.c_int), ("length", ctypes.c_int * 3),
                ("tau", ctypes.c_double), ("tau_mrt", ctypes.c_double * 15),
                ("c_smag", ctypes.c_double), ("collision_type", ctypes.c_int),
                ("forcing", ctypes.c_int), ("macro_bc", ctypes.c_int),
                ("micro_bc", ctypes.c_int), ("init_type", ctypes.c_int),
                ("tolerance", ctypes.c_double), ("h", ctypes.c_int), ("dt", ctypes.c_int),
                ("storage", ctypes.c_int), ("streaming", ctypes.c_int),
                ("compat", ctypes.c_uint), ("storage_scale", ctypes.c_double),
                ("device", ctypes.c_int), ("block_size", ctypes.c_int),
                ("kernel", ctypes.c_int), ("reserved", ctypes.c_int * 5)]


class Domain(ctypes.Structure):
    _fields_ = [("geometry", _DP), ("force", _DP * 3), ("macro_bc", _IP),
                ("micro_bc", _IP), ("u", _DP * 3), ("rho", _DP), ("f", _DP)]


class Diag(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("momentum", ctypes.c_double * 3),
                ("kinetic_energy", ctypes.c_double), ("step", ctypes.c_longlong),
                ("nonfinite", ctypes.c_int), ("valid", ctypes.c_int)]


class LbmcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"lbmc status {status}: {message}")
        self.status = status


_lib = None


PATH_MAX = 256


class RunConfig(ctypes.Structure):
    """lbmc_run_config: what an input file sets (include/lbmc.h)."""
    _fields_ = [("cfg", Config), ("project_name", ctypes.c_char * PATH_MAX),
                ("domain_file", ctypes.c_char * PATH_MAX), ("output_file", ctypes.c_char * PATH_MAX),
                ("max_t", ctypes.c_int), ("file_out", ctypes.c_int), ("screen_mes", ctypes.c_int),
                ("steady_check", ctypes.c_int), ("output_u", ctypes.c_int * 3),
                ("output_rho", ctypes.c_int), ("output_pressure", ctypes.c_int),
                ("screen_node", ctypes.c_int * 3), ("interactive", ctypes.c_int),
                ("lz_given", ctypes.c_int), ("lattice_given", ctypes.c_int),
                ("tau_mrt_count", ctypes.c_int)]


class RunResult(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("steady", ctypes.c_int), ("nonfinite", ctypes.c_int),
                ("outputs", ctypes.c_int), ("residual", ctypes.c_double * 3), ("seconds", ctypes.c_double)]


def library() -> ctypes.CDLL:
    """The in-tree liblbmc.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C lbm-c_b200` "
                               "(the engine has no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        lib.lbmc_config_default.argtypes = [ctypes.POINTER(Config), ctypes.c_int]
        lib.lbmc_validate.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(Domain)]
        lib.lbmc_init.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(Domain),
                                  ctypes.POINTER(_P)]
        lib.lbmc_iterate.argtypes = [_P, ctypes.c_int, ctypes.c_uint]
        lib.lbmc_fetch.argtypes = [_P, ctypes.c_int, _P, ctypes.c_size_t]
        lib.lbmc_destroy.argtypes = [_P]
        lib.lbmc_get_step.argtypes = [_P, ctypes.POINTER(ctypes.c_longlong)]
        lib.lbmc_set_stream.argtypes = [_P, _P]
        lib.lbmc_synchronize.argtypes = [_P]
        lib.lbmc_status_string.restype = ctypes.c_char_p
        lib.lbmc_status_string.argtypes = [ctypes.c_int]
        lib.lbmc_last_error.restype = ctypes.c_char_p
        lib.lbmc_last_error.argtypes = []
        lib.lbmc_classify.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(Domain), _P, _P,
                                      ctypes.POINTER(ctypes.c_int)]
        lib.lbmc_lattice_tables.argtypes = [ctypes.c_int, _P, _P, _P, _P]
        lib.lbmc_selftest_wait_timeout.argtypes = [ctypes.c_int, ctypes.c_double]
        lib.lbmc_selftest_wait_timeout.restype = ctypes.c_int
        lib.lbmc_macro_sums_noalloc.argtypes = [ctypes.c_int, _P, _P, _P, _P, ctypes.c_longlong,
                                                _P, _P]
        lib.lbmc_macro_sums_noalloc.restype = ctypes.c_int
        lib.lbmc_probe.argtypes = [_P, ctypes.c_longlong, _P]
        lib.lbmc_read_input.argtypes = [ctypes.c_char_p, ctypes.POINTER(RunConfig), ctypes.c_char_p,
                                        ctypes.c_size_t]
        lib.lbmc_model_build.argtypes = [ctypes.POINTER(RunConfig), ctypes.POINTER(_P)]
        lib.lbmc_model_domain.argtypes = [_P, ctypes.POINTER(Domain)]
        lib.lbmc_model_free.argtypes = [_P]
        lib.lbmc_model_free.restype = None
        lib.lbmc_output_open.argtypes = [ctypes.c_char_p, ctypes.c_int, _P, ctypes.POINTER(_P)]
        lib.lbmc_output_append.argtypes = [_P, ctypes.c_longlong, ctypes.c_int, _P, _P]
        lib.lbmc_output_close.argtypes = [_P]
        lib.lbmc_run.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config), ctypes.c_int,
                                 ctypes.POINTER(RunResult)]
        for name in ("lbmc_config_default", "lbmc_validate", "lbmc_init", "lbmc_iterate",
                     "lbmc_fetch", "lbmc_destroy", "lbmc_get_step", "lbmc_set_stream",
                     "lbmc_synchronize", "lbmc_classify", "lbmc_lattice_tables", "lbmc_probe",
                     "lbmc_read_input", "lbmc_model_build", "lbmc_model_domain", "lbmc_output_open",
                     "lbmc_output_append", "lbmc_output_close", "lbmc_run"):
            getattr(lib, name).restype = ctypes.c_int
        _lib = lib
    return _lib


def check(status: int):
    if status != OK:
        raise LbmcError(status, library().lbmc_last_error().decode())


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions include/lbmc.h declares."""
    import re
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbmc_[a-z_]+)\s*\(", text)))


def _as_f64(a, n):
    return None if a is None else np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1)[:n])


class _Keep:
    """Holds the numpy arrays a Domain points into."""

    def __init__(self):
        self.arrays = []

    def ptr_d(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, np.float64)
        self.arrays.append(a)
        return a.ctypes.data_as(_DP)

    def ptr_i(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, np.int32)
        self.arrays.append(a)
        return a.ctypes.data_as(_IP)


def make_config(lattice, length, tau=1.0, tau_mrt=(), c_smag=0.0, collision_type=BGK,
                forcing=False, macro_bc=False, micro_bc=False, init_type=INIT_STATIC,
                storage=F32, compat=0, storage_scale=0.0, device=0, streaming=STREAM_SHIFT,
                tolerance=0.0, kernel=KERNEL_AUTO) -> Config:
    lat = LATTICE_IDS.get(lattice, lattice)
    cfg = Config()
    check(library().lbmc_config_default(ctypes.byref(cfg), lat))
    for d in range(3):
        cfg.length[d] = int(length[d]) if d < len(length) else 1
    if lat == D2Q9:
        cfg.length[2] = 1
    cfg.tau = tau
    for i, v in enumerate(tau_mrt):
        cfg.tau_mrt[i] = v
    cfg.c_smag = c_smag
    cfg.collision_type = collision_type
    cfg.forcing = int(bool(forcing))
    cfg.macro_bc = int(bool(macro_bc))
    cfg.micro_bc = int(bool(micro_bc))
    cfg.init_type = init_type
    cfg.storage = STORAGE_IDS.get(storage, storage)
    cfg.compat = compat
    cfg.storage_scale = storage_scale
    cfg.device = device
    cfg.streaming = streaming
    cfg.tolerance = tolerance
    cfg.kernel = kernel
    return cfg


def make_domain(n, dim, q, geometry=None, force=None, macro=None, micro=None, u=None,
                rho=None, f=None):
    keep = _Keep()
    dom = Domain()
    dom.geometry = keep.ptr_d(geometry)
    for d in range(3):
        dom.force[d] = keep.ptr_d(None if force is None or d >= dim else np.asarray(force)[d])
        dom.u[d] = keep.ptr_d(None if u is None or d >= dim else np.asarray(u)[d])
    dom.macro_bc = keep.ptr_i(macro)
    dom.micro_bc = keep.ptr_i(micro)
    dom.rho = keep.ptr_d(rho)
    dom.f = keep.ptr_d(f)
    return dom, keep


def _checked_out(out, shape):
    if not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.shape == shape
            and out.flags.c_contiguous):
        raise ValueError(f"out must be a C-contiguous float64 array of shape {shape}")
    return out


class Engine:
    """One lbmc handle: ``Engine(cfg, domain)`` = lbmc_init."""

    def __init__(self, cfg: Config, dom: Domain):
        lib = library()
        self.cfg = cfg
        self.dim = 2 if cfg.lattice == D2Q9 else 3
        self.q = 9 if cfg.lattice == D2Q9 else 15
        self.n = int(np.prod([cfg.length[d] for d in range(self.dim)]))
        h = _P()
        check(lib.lbmc_init(ctypes.byref(cfg), ctypes.byref(dom), ctypes.byref(h)))
        self.h = h

    @classmethod
    def from_case(cls, case, storage=F32, init_type=None, compat=None, **kw):
        """Builds an engine for an oracle ``Case`` (tests/cases.py)."""
        a = case.arrays()
        if init_type is None:
            init_type = INIT_F if a["f0"] is not None else INIT_STATIC
        cfg = make_config(case.lattice, case.length, tau=case.tau, tau_mrt=case.tau_mrt,
                          c_smag=case.c_smag, collision_type=case.collision_type,
                          forcing=case.forcing, macro_bc=case.macro_bc,
                          micro_bc=case.micro_bc, init_type=init_type, storage=storage,
                          compat=case.compat if compat is None else compat, **kw)
        dom, keep = make_domain(case.n, case.dim, case.q, a["geometry"], a["force"], a["macro"],
                                a["micro"], a["u"], a["rho"], a["f0"])
        eng = cls(cfg, dom)
        del keep
        return eng

    def iterate(self, nsteps: int, flags: int = 0):
        check(library().lbmc_iterate(self.h, nsteps, flags))

    def _fetch(self, field, out):
        check(library().lbmc_fetch(self.h, field, out.ctypes.data_as(_P), out.nbytes))
        return out

    def rho(self, out=None):
        """rho per node (FP64); `out`, if given, is filled and returned."""
        if out is None:
            out = np.empty(self.n)
        return self._fetch(FIELD_RHO, _checked_out(out, (self.n,)))

    def u(self, out=None):
        """u per node, shape (dim, n) (FP64); `out`, if given, is filled and returned."""
        if out is None:
            out = np.empty((self.dim, self.n))
        _checked_out(out, (self.dim, self.n))
        for d in range(self.dim):
            self._fetch(FIELD_U_X + d, out[d])
        return out

    def f(self):
        return self._fetch(FIELD_F, np.empty((self.q, self.n)))

    def diag(self) -> Diag:
        d = Diag()
        check(library().lbmc_fetch(self.h, FIELD_DIAG, ctypes.cast(ctypes.byref(d), _P),
                                   ctypes.sizeof(d)))
        return d

    def step(self) -> int:
        v = ctypes.c_longlong()
        check(library().lbmc_get_step(self.h, ctypes.byref(v)))
        return v.value

    def synchronize(self):
        check(library().lbmc_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            library().lbmc_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------- batched domains

class BatchConfig(ctypes.Structure):
    _fields_ = [("tau", ctypes.c_double), ("force", ctypes.c_double * 2),
                ("collision_type", ctypes.c_int), ("storage", ctypes.c_int),
                ("storage_scale", ctypes.c_double), ("device", ctypes.c_int),
                ("block_threads", ctypes.c_int), ("steps_per_launch", ctypes.c_int),
                ("wide_min_nodes", ctypes.c_int), ("wide_below", ctypes.c_int),
                ("reserved", ctypes.c_int * 6)]


class BatchDomain(ctypes.Structure):
    _fields_ = [("length", ctypes.c_int * 2), ("geometry", _DP)]


class BatchResult(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("delta_u", ctypes.c_double),
                ("elapsed_ms", ctypes.c_double), ("converged", ctypes.c_int),
                ("nonfinite", ctypes.c_int)]


def _batch_lib():
    lib = library()
    if not getattr(lib, "_batch_ready", False):
        lib.lbmc_batch_init.argtypes = [ctypes.POINTER(BatchConfig), ctypes.c_int,
                                        ctypes.POINTER(BatchDomain), ctypes.POINTER(_P)]
        lib.lbmc_batch_run.argtypes = [_P, ctypes.c_longlong, ctypes.c_double, ctypes.c_int,
                                       ctypes.POINTER(BatchResult)]
        lib.lbmc_batch_fetch.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_size_t]
        lib.lbmc_batch_info.argtypes = [_P, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
        lib.lbmc_batch_destroy.argtypes = [_P]
        for name in ("lbmc_batch_init", "lbmc_batch_run", "lbmc_batch_fetch",
                     "lbmc_batch_info", "lbmc_batch_destroy"):
            getattr(lib, name).restype = ctypes.c_int
        lib._batch_ready = True
    return lib


class Batch:
    """Many independent D2Q9 domains in one persistent launch (lbmc_batch_*)."""

    def __init__(self, geometries, tau=1.0, force=(1e-6, 0.0), collision_type=NTPOR,
                 storage=F16, storage_scale=0.0, device=0, block_threads=0, steps_per_launch=0,
                 wide_below=0, wide_min_nodes=0):
        lib = _batch_lib()
        cfg = BatchConfig()
        cfg.tau = tau
        cfg.force[0], cfg.force[1] = force
        cfg.collision_type = collision_type
        cfg.storage = STORAGE_IDS.get(storage, storage)
        cfg.storage_scale = storage_scale
        cfg.device = device
        cfg.block_threads = block_threads
        cfg.steps_per_launch = steps_per_launch
        cfg.wide_below = wide_below
        cfg.wide_min_nodes = wide_min_nodes
        self._keep = []
        doms = (BatchDomain * len(geometries))()
        self.shapes = []
        for d, g in enumerate(geometries):
            g = np.ascontiguousarray(g, np.float64)
            ly, lx = g.shape
            doms[d].length[0], doms[d].length[1] = lx, ly
            doms[d].geometry = g.ctypes.data_as(_DP)
            self._keep.append(g)
            self.shapes.append((ly, lx))
        h = _P()
        check(lib.lbmc_batch_init(ctypes.byref(cfg), len(geometries), doms, ctypes.byref(h)))
        self.h, self.n = h, len(geometries)

    def run(self, max_steps, tol, check_every=100):
        """Per-domain results.  A domain that became non-finite raises
        LbmcError(ERR_NAN) whose ``results`` attribute holds them all."""
        res = (BatchResult * self.n)()
        status = _batch_lib().lbmc_batch_run(self.h, max_steps, tol, check_every, res)
        if status == ERR_NAN:
            err = LbmcError(status, library().lbmc_last_error().decode())
            err.results = res
            raise err
        check(status)
        return res

    def fetch(self, d, field):
        ly, lx = self.shapes[d]
        out = np.empty((9 if field == FIELD_F else 1) * lx * ly)
        check(_batch_lib().lbmc_batch_fetch(self.h, d, field, out.ctypes.data_as(_P), out.nbytes))
        return out.reshape(9, -1) if field == FIELD_F else out

    def info(self):
        tot, th, st, res = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(_batch_lib().lbmc_batch_info(self.h, ctypes.byref(tot), ctypes.byref(th),
                                           ctypes.byref(st), ctypes.byref(res)))
        return dict(total_nodes=tot.value, threads=th.value, steps_per_launch=st.value,
                    resident_domains=res.value)

    def close(self):
        if getattr(self, "h", None):
            _batch_lib().lbmc_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ learned closure

MLP_PARAMS = 1313


def _mlp_lib():
    lib = library()
    if not getattr(lib, "_mlp_ready", False):
        lib.lbmc_mlp_create.argtypes = [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(_P)]
        lib.lbmc_mlp_set_normalization.argtypes = [_P, _P, _P, _P, _P, ctypes.c_float]
        lib.lbmc_mlp_features.argtypes = [ctypes.c_int, _P, _P, ctypes.c_longlong, _P]
        lib.lbmc_mlp_train.argtypes = [_P, _P, _P, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, _P]
        lib.lbmc_mlp_gradients.argtypes = [_P, _P, _P, ctypes.c_longlong, _P,
                                           ctypes.POINTER(ctypes.c_float)]
        lib.lbmc_mlp_predict.argtypes = [_P, _P, ctypes.c_longlong, _P]
        lib.lbmc_mlp_predict_step.argtypes = [_P, _P, ctypes.c_longlong, _P]
        lib.lbmc_mlp_get_params.argtypes = [_P, _P]
        lib.lbmc_mlp_set_params.argtypes = [_P, _P]
        lib.lbmc_mlp_destroy.argtypes = [_P]
        lib.lbmc_set_closure.argtypes = [_P, _P, ctypes.c_int]
        for name in ("lbmc_mlp_create", "lbmc_mlp_set_normalization", "lbmc_mlp_features",
                     "lbmc_mlp_train", "lbmc_mlp_gradients", "lbmc_mlp_predict", "lbmc_mlp_predict_step",
                     "lbmc_mlp_get_params", "lbmc_mlp_set_params", "lbmc_mlp_destroy",
                     "lbmc_set_closure"):
            getattr(lib, name).restype = ctypes.c_int
        lib._mlp_ready = True
    return lib


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, np.float32)
    return a if shape is None else a.reshape(shape)


def mlp_features(strain6, rho=None, device=0):
    """Six closure inputs per sample from strain tensors (n, 6) and densities."""
    S = _f32(strain6, (-1, 6))
    n = S.shape[0]
    r = None if rho is None else _f32(rho, (n,))
    out = np.empty((n, 6), np.float32)
    check(_mlp_lib().lbmc_mlp_features(device, S.ctypes.data, None if r is None else r.ctypes.data,
                                       n, out.ctypes.data))
    return out


class Mlp:
    """The closure network (lbmc_mlp_*)."""

    def __init__(self, seed=0, device=0):
        h = _P()
        check(_mlp_lib().lbmc_mlp_create(device, seed, ctypes.byref(h)))
        self.h = h

    def set_normalization(self, mean, std, lo=None, hi=None, target_scale=1.0):
        m, s = _f32(mean), _f32(std)
        lo = None if lo is None else _f32(lo)
        hi = None if hi is None else _f32(hi)
        self._norm = (m, s, lo, hi)
        check(_mlp_lib().lbmc_mlp_set_normalization(
            self.h, m.ctypes.data, s.ctypes.data, None if lo is None else lo.ctypes.data,
            None if hi is None else hi.ctypes.data, target_scale))

    def train(self, features, target, epochs=10, batch=4096, lr=1e-3):
        X, y = _f32(features, (-1, 6)), _f32(target, (-1,))
        hist = np.zeros(epochs, np.float32)
        check(_mlp_lib().lbmc_mlp_train(self.h, X.ctypes.data, y.ctypes.data, X.shape[0], epochs,
                                        batch, lr, hist.ctypes.data))
        return hist

    def gradients(self, features, target):
        X, y = _f32(features, (-1, 6)), _f32(target, (-1,))
        g = np.empty(MLP_PARAMS, np.float32)
        loss = ctypes.c_float()
        check(_mlp_lib().lbmc_mlp_gradients(self.h, X.ctypes.data, y.ctypes.data, X.shape[0],
                                            g.ctypes.data, ctypes.byref(loss)))
        return g, loss.value

    def predict(self, features):
        X = _f32(features, (-1, 6))
        out = np.empty(X.shape[0], np.float32)
        check(_mlp_lib().lbmc_mlp_predict(self.h, X.ctypes.data, X.shape[0], out.ctypes.data))
        return out

    def predict_step(self, features):
        """The prediction as the step computes it (tensor cores, BF16 activations)."""
        X = _f32(features, (-1, 6))
        out = np.empty(X.shape[0], np.float32)
        check(_mlp_lib().lbmc_mlp_predict_step(self.h, X.ctypes.data, X.shape[0], out.ctypes.data))
        return out

    def params(self):
        p = np.empty(MLP_PARAMS, np.float32)
        check(_mlp_lib().lbmc_mlp_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = _f32(p)
        check(_mlp_lib().lbmc_mlp_set_params(self.h, p.ctypes.data))

    def attach(self, engine, iterations=2):
        check(_mlp_lib().lbmc_set_closure(engine.h, self.h, iterations))

    def close(self):
        if getattr(self, "h", None):
            _mlp_lib().lbmc_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------- run control

def read_input(path):
    """lbmc_read_input: (RunConfig, the reader's report)."""
    rc = RunConfig()
    echo = ctypes.create_string_buffer(1 << 16)
    check(library().lbmc_read_input(os.fsencode(path), ctypes.byref(rc), echo, len(echo)))
    return rc, echo.value.decode()


def run(path, storage=F32, streaming=STREAM_AA, device=0, quiet=True):
    """lbmc_run: the reference's driver loop on an input file; returns
    (status, RunResult).  LBMC_ERR_NAN is returned, not raised."""
    ov = Config()
    check(library().lbmc_config_default(ctypes.byref(ov), D2Q9))
    ov.storage = STORAGE_IDS.get(storage, storage)
    ov.streaming = streaming
    ov.device = device
    res = RunResult()
    st = library().lbmc_run(os.fsencode(path), ctypes.byref(ov), int(quiet), ctypes.byref(res))
    if st not in (OK, ERR_NAN):
        check(st)
    return st, res


class Output:
    """lbmc_output_*: the CGNS-structured solution writer."""

    def __init__(self, path, dim, length):
        h = _P()
        L = (ctypes.c_int * 3)(*(list(length) + [1] * (3 - len(length))))
        check(library().lbmc_output_open(os.fsencode(path), dim, L, ctypes.byref(h)))
        self.h = h

    def append(self, step, fields):
        """fields: {label: float64 array of N values}."""
        arrs = [np.ascontiguousarray(v, np.float64) for v in fields.values()]
        data = (_P * len(arrs))(*[a.ctypes.data for a in arrs])
        labels = (ctypes.c_char_p * len(arrs))(*[k.encode() for k in fields])
        check(library().lbmc_output_append(self.h, step, len(arrs), data, labels))

    def close(self):
        if self.h:
            check(library().lbmc_output_close(self.h))
            self.h = None
