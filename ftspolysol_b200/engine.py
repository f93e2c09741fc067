"""Python front end of libftsp.so (the engine's C ABI, include/ftsp.h).

Mirrors the reference's step-loop surface: compute_densities
(complexLangevin.cu:255-260), measure (observable.cu:53-67), step
(complexLangevin.cu:669-698), the deviceState field names
(deviceState.h:6-48).  The CUDA library is the only implementation: if it
cannot be loaded, or no CUDA device is present, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libftsp.so")

FTSP_OK, FTSP_NONFINITE, FTSP_ERROR, FTSP_TIMEOUT = 0, 1, 2, 3
FP64, FP32 = 0, 1
SCHEME_PC, SCHEME_SI = 0, 1
STRESS_NAMES = ("xx", "yy", "zz", "xy", "xz", "yz")


class FtspError(RuntimeError):
    pass


class NonFinite(RuntimeError):
    pass


class ftsp_config(C.Structure):
    _fields_ = [
        ("m1", C.c_int), ("m2", C.c_int), ("m3", C.c_int),
        ("L1", C.c_double), ("L2", C.c_double), ("L3", C.c_double),
        ("dV", C.c_double), ("a", C.c_double), ("lB", C.c_double), ("dt", C.c_double),
        ("lambda_psi", C.c_double),
        ("M", C.c_int), ("n_modes", C.c_int),
        ("mode_coeff", C.POINTER(C.c_double)), ("mode_gamma", C.POINTER(C.c_double)),
        ("mode_O", C.POINTER(C.c_double)), ("mode_lambda", C.POINTER(C.c_double)),
        ("n_species", C.c_int), ("num_chains", C.POINTER(C.c_double)), ("N", C.POINTER(C.c_int)),
        ("seg_type", C.POINTER(C.c_int)), ("seg_charge", C.POINTER(C.c_double)),
        ("seg_bond", C.POINTER(C.c_double)),
        ("n_ions", C.c_int), ("ion_valence", C.POINTER(C.c_double)), ("ion_count", C.POINTER(C.c_double)),
        ("ion_smear", C.POINTER(C.c_double)),
        ("self_pressure", C.c_double), ("stress_mask", C.c_int), ("isotropic_pressure", C.c_int),
        ("noise", C.c_int), ("seed", C.c_ulonglong), ("precision", C.c_int), ("scheme", C.c_int),
        ("device", C.c_int), ("restart_interval", C.c_int), ("autotune", C.c_int),
        ("max_restarts", C.c_int),
    ]


class ftsp_views(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("omega", "psi", "omega_bar", "psi_bar", "rho_type", "rho_p", "rho_c",
                                          "rho_c_poly", "rho_c_ion", "ion_rho", "drift", "drift_bar", "dpsi",
                                          "dpsi_bar")]


class ftsp_kernel_stat(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("ms", C.c_double), ("launches", C.c_longlong), ("bytes", C.c_double)]


class ftsp_tune_info(C.Structure):
    _fields_ = [("tuned", C.c_int), ("cached", C.c_int), ("compile_time", C.c_int), ("max_radix", C.c_int),
                ("tile_width", C.c_int), ("candidates", C.c_int), ("best_ms", C.c_double), ("default_ms", C.c_double)]


class ftsp_learn_config(C.Structure):
    _fields_ = [("N", C.c_double), ("lB", C.c_double), ("salt", C.c_double), ("lr", C.c_double), ("batch", C.c_int),
                ("refresh_every", C.c_int), ("fallback_ratio", C.c_double), ("seed", C.c_ulonglong)]


class ftsp_learn_stats(C.Structure):
    _fields_ = [("collected", C.c_longlong), ("checks", C.c_longlong), ("fallbacks", C.c_longlong),
                ("residual_learned", C.c_double), ("residual_analytic", C.c_double),
                ("residual_learned_sum", C.c_double), ("residual_analytic_sum", C.c_double), ("loss", C.c_double),
                ("iterations", C.c_int), ("using_learned", C.c_int), ("n_params", C.c_int),
                ("valid_targets", C.c_longlong)]


_lib = None


def library_path() -> str:
    return LIB_PATH


def lib():
    """Loads libftsp.so (building it first if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.ftsp_create.argtypes = [C.POINTER(ftsp_config), C.POINTER(vp)]
        L.ftsp_destroy.argtypes = [vp]
        L.ftsp_last_error.restype = C.c_char_p
        L.ftsp_last_error.argtypes = [vp]
        L.ftsp_set_stream.argtypes = [vp, vp]
        L.ftsp_set_fields.argtypes = [vp, vp, vp]
        L.ftsp_set_fields_async.argtypes = [vp, vp, vp]
        L.ftsp_get_field.argtypes = [vp, C.c_char_p, vp, C.POINTER(C.c_longlong)]
        L.ftsp_compute_densities.argtypes = [vp, C.c_int, vp]
        L.ftsp_record_length.argtypes = [vp]
        L.ftsp_measure.argtypes = [vp, C.c_int, vp]
        L.ftsp_set_noise.argtypes = [vp, vp]
        L.ftsp_set_seed.argtypes = [vp, C.c_ulonglong]
        L.ftsp_step.argtypes = [vp, vp, vp, vp]
        L.ftsp_step_async.argtypes = [vp]
        L.ftsp_read_status.argtypes = [vp, vp, vp]
        L.ftsp_state_views.argtypes = [vp, C.POINTER(ftsp_views)]
        L.ftsp_last_launch_count.restype = C.c_longlong
        L.ftsp_last_launch_count.argtypes = [vp]
        L.ftsp_propagate_chain.argtypes = [vp, vp, C.c_int, C.c_double, vp, vp]
        L.ftsp_restart_count.restype = C.c_longlong
        L.ftsp_restart_count.argtypes = [vp]
        L.ftsp_rollback_info.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
        L.ftsp_average_start.argtypes = [vp, C.c_int, C.c_longlong, C.c_int]
        L.ftsp_average_read.argtypes = [vp, vp, vp, C.POINTER(C.c_longlong)]
        L.ftsp_propagate_chain_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                                   vp, C.c_int, C.c_double, vp, vp, vp]
        L.ftsp_profile_enable.argtypes = [vp, C.c_int]
        L.ftsp_profile_read.argtypes = [vp, C.POINTER(ftsp_kernel_stat), C.c_int, C.POINTER(C.c_int)]
        L.ftsp_set_dt.argtypes = [vp, C.c_double]
        L.ftsp_set_adaptive.argtypes = [vp, C.c_double]
        L.ftsp_set_chain_symmetry.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        L.ftsp_set_step_graph.argtypes = [vp, C.c_int]
        L.ftsp_step_info.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ftsp_tune_info_get.argtypes = [vp, C.POINTER(ftsp_tune_info)]
        L.ftsp_learn_configure.argtypes = [vp, C.POINTER(ftsp_learn_config)]
        L.ftsp_learn_collect.argtypes = [vp, C.c_int]
        L.ftsp_learn_reset.argtypes = [vp]
        L.ftsp_learn_train.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        L.ftsp_learn_use.argtypes = [vp, C.c_int]
        L.ftsp_learn_get_stats.argtypes = [vp, C.POINTER(ftsp_learn_stats)]
        L.ftsp_learn_get_weights.argtypes = [vp, vp, C.POINTER(C.c_int)]
        L.ftsp_learn_set_weights.argtypes = [vp, vp, C.c_int]
        L.ftsp_learn_grad.argtypes = [vp, vp, vp, vp, C.c_int, C.POINTER(C.c_double), vp]
        L.ftsp_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.POINTER(vp)]
        L.ftsp_batch_step.argtypes = [vp, C.c_int]
        L.ftsp_batch_sync.argtypes = [vp]
        L.ftsp_batch_stream.restype = vp
        L.ftsp_batch_stream.argtypes = [vp]
        L.ftsp_batch_launch_count.restype = C.c_longlong
        L.ftsp_batch_launch_count.argtypes = [vp]
        L.ftsp_batch_last_error.restype = C.c_char_p
        L.ftsp_batch_last_error.argtypes = [vp]
        L.ftsp_batch_destroy.restype = None
        L.ftsp_batch_destroy.argtypes = [vp]
        _lib = L
    return _lib


# exported symbols of include/ftsp.h
ABI_SYMBOLS = ("ftsp_create", "ftsp_destroy", "ftsp_last_error", "ftsp_set_stream", "ftsp_set_fields",
               "ftsp_set_fields_async",
               "ftsp_get_field", "ftsp_compute_densities", "ftsp_record_length", "ftsp_measure",
               "ftsp_set_noise", "ftsp_set_seed", "ftsp_step", "ftsp_step_async", "ftsp_read_status",
               "ftsp_state_views", "ftsp_last_launch_count", "ftsp_profile_enable", "ftsp_profile_read",
               "ftsp_propagate_chain", "ftsp_propagate_chain_noalloc", "ftsp_restart_count", "ftsp_rollback_info",
               "ftsp_average_start", "ftsp_average_read",
               "ftsp_set_dt",
               "ftsp_tune_info_get", "ftsp_set_adaptive", "ftsp_step_info", "ftsp_set_chain_symmetry", "ftsp_set_step_graph",
               "ftsp_learn_configure", "ftsp_learn_collect", "ftsp_learn_reset", "ftsp_learn_train", "ftsp_learn_use",
               "ftsp_learn_get_stats", "ftsp_learn_get_weights", "ftsp_learn_set_weights", "ftsp_learn_grad",
               "ftsp_batch_create", "ftsp_batch_step", "ftsp_batch_sync", "ftsp_batch_stream",
               "ftsp_batch_launch_count", "ftsp_batch_last_error", "ftsp_batch_destroy")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def propagate_chain_noalloc(m, L, w_ptr: int, N: int, bond_length: float, q_end_ptr: int, stream: int = 0):
    """Chain propagation that allocates no device memory (no handle needed).

    For callers that cannot allocate: under a framework that owns the device
    memory pool, or in loops that must not wait on the allocator.  w and
    q_end are device pointers to m1*m2*m3 complex128 values; at most 64^3
    points and 256 per axis.  The call is synchronous (it waits for the
    stream and returns Q on the host).  Do not run calls concurrently from
    several threads: they share one scratch array, tables included.
    Returns (status, Q)."""
    Q = np.zeros(2)
    rc = lib().ftsp_propagate_chain_noalloc(int(m[0]), int(m[1]), int(m[2]), float(L[0]), float(L[1]), float(L[2]),
                                            C.c_void_p(w_ptr), int(N), float(bond_length), C.c_void_p(q_end_ptr),
                                            Q.ctypes.data, C.c_void_p(stream))
    return rc, complex(Q[0], Q[1])


def last_error() -> str:
    """Error text of the last failed handle-less call on this thread."""
    return (lib().ftsp_last_error(None) or b"").decode()


class Engine:
    """One complex-Langevin system on one GPU.

    `derived` holds the derived parameters (the output of the host-side
    param/sequence/ion setup): m, L, dV, a, lB, dt, lambda_psi, M, modes
    [{coeff, lambda, gamma, O}], species [{num_chains, types, charges,
    bonds}], ions [{valence, count, smear}], self_pressure, stress (component
    names), isotropic_pressure.
    """

    def __init__(self, derived: dict, precision: int = FP64, scheme: int = SCHEME_PC, noise: bool = False,
                 seed: int = 0, device: int = 0, restart_interval: int = 0, autotune: bool = False,
                 max_restarts: int = 20):
        L = lib()
        self._keep = []

        def arr(x, dt=np.float64):
            a = np.ascontiguousarray(np.asarray(x, dtype=dt))
            if a.size == 0:
                a = np.zeros(1, dtype=dt)
            self._keep.append(a)
            return a

        d = derived
        self.m = tuple(int(v) for v in d["m"])
        self.size = int(np.prod(self.m))
        modes = d["modes"]
        self.n_modes = len(modes)
        self.M = int(d["M"])
        sp = d["species"]
        self.n_species = len(sp)
        self.n_ions = len(d["ions"])
        cfg = ftsp_config()
        cfg.m1, cfg.m2, cfg.m3 = self.m
        cfg.L1, cfg.L2, cfg.L3 = [float(v) for v in d["L"]]
        cfg.dV = float(d["dV"])
        cfg.a = float(d["a"])
        cfg.lB = float(d["lB"])
        cfg.dt = float(d["dt"])
        cfg.lambda_psi = float(d["lambda_psi"])
        cfg.M = self.M
        cfg.n_modes = self.n_modes
        cfg.mode_coeff = _dp(arr([m["coeff"] for m in modes]))
        g = []
        for m in modes:
            g += [complex(m["gamma"]).real, complex(m["gamma"]).imag]
        cfg.mode_gamma = _dp(arr(g))
        cfg.mode_O = _dp(arr([o for m in modes for o in m["O"]]))
        cfg.mode_lambda = _dp(arr([m["lambda"] for m in modes]))
        cfg.n_species = len(sp)
        cfg.num_chains = _dp(arr([s["num_chains"] for s in sp]))
        cfg.N = _ip(arr([len(s["types"]) for s in sp], np.int32))
        cfg.seg_type = _ip(arr([t for s in sp for t in s["types"]], np.int32))
        cfg.seg_charge = _dp(arr([q for s in sp for q in s["charges"]]))
        cfg.seg_bond = _dp(arr([b for s in sp for b in s["bonds"]]))
        ions = d["ions"]
        cfg.n_ions = len(ions)
        cfg.ion_valence = _dp(arr([i["valence"] for i in ions]))
        cfg.ion_count = _dp(arr([i["count"] for i in ions]))
        cfg.ion_smear = _dp(arr([i["smear"] for i in ions]))
        cfg.self_pressure = float(d["self_pressure"])
        mask = 0
        for c in d.get("stress", ()):
            mask |= 1 << STRESS_NAMES.index(c)
        cfg.stress_mask = mask
        cfg.isotropic_pressure = int(bool(d.get("isotropic_pressure", False)))
        cfg.noise = int(bool(noise))
        cfg.seed = int(seed)
        cfg.precision = int(precision)
        cfg.scheme = int(scheme)
        cfg.device = int(device)
        cfg.restart_interval = int(restart_interval)
        cfg.max_restarts = int(max_restarts)
        cfg.autotune = int(bool(autotune))
        self.precision = precision
        self._cfg = cfg
        h = C.c_void_p()
        rc = L.ftsp_create(C.byref(cfg), C.byref(h))
        if rc != FTSP_OK:
            raise FtspError("ftsp_create failed: " + (L.ftsp_last_error(None) or b"").decode())
        self.h = h
        self.record_len = L.ftsp_record_length(self.h)

    # ---- helpers ----
    def _check(self, rc, what):
        if rc == FTSP_OK:
            return rc
        if rc == FTSP_NONFINITE:
            raise NonFinite(what + ": non-finite value")
        raise FtspError(what + ": " + (lib().ftsp_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            lib().ftsp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- API ----
    def set_fields(self, omega, psi):
        o = np.ascontiguousarray(np.asarray(omega, dtype=np.complex128).reshape(self.n_modes, self.size))
        p = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128).reshape(self.size))
        if o.size == 0:
            o = np.zeros(1, dtype=np.complex128)
        self._check(lib().ftsp_set_fields(self.h, o.ctypes.data, p.ctypes.data), "set_fields")

    def get(self, name: str) -> np.ndarray:
        n = C.c_longlong(0)
        self._check(lib().ftsp_get_field(self.h, name.encode(), None, C.byref(n)), "get_field")
        out = np.zeros(max(1, n.value), dtype=np.float64)
        self._check(lib().ftsp_get_field(self.h, name.encode(), out.ctypes.data, C.byref(n)), "get_field")
        return out[: n.value].view(np.complex128).reshape(-1, self.size)

    def compute_densities(self, which: int = 0) -> np.ndarray:
        Q = np.zeros(max(1, self.n_species), dtype=np.complex128)
        self._check(lib().ftsp_compute_densities(self.h, which, Q.ctypes.data), "compute_densities")
        return Q[: self.n_species]

    def measure(self, which: int = 0) -> np.ndarray:
        rec = np.zeros(self.record_len, dtype=np.complex128)
        self._check(lib().ftsp_measure(self.h, which, rec.ctypes.data), "measure")
        return rec

    def set_fields_ptr(self, omega_ptr: int, psi_ptr: int):
        """set_fields from raw host pointers (e.g. pinned buffers)."""
        self._check(lib().ftsp_set_fields(self.h, C.c_void_p(omega_ptr), C.c_void_p(psi_ptr)), "set_fields")

    def set_fields_async_ptr(self, omega_ptr: int, psi_ptr: int):
        """Upload of new fields from (pinned) host memory that overlaps the
        step in flight; installed by the next call that uses the fields.
        The host buffers must stay unchanged until results have been read."""
        self._check(lib().ftsp_set_fields_async(self.h, C.c_void_p(omega_ptr), C.c_void_p(psi_ptr)), "set_fields_async")

    def propagate_chain(self, w_ptr: int, N: int, bond_length: float, q_end_ptr: int) -> complex:
        """Chain propagation in an external field (device pointers, complex128)."""
        Q = np.zeros(2)
        self._check(lib().ftsp_propagate_chain(self.h, C.c_void_p(w_ptr), int(N), float(bond_length),
                                               C.c_void_p(q_end_ptr), Q.ctypes.data), "propagate_chain")
        return complex(Q[0], Q[1])

    def profile(self, on: bool = True):
        self._check(lib().ftsp_profile_enable(self.h, int(on)), "profile_enable")

    def profile_read(self) -> dict:
        n = C.c_int(0)
        self._check(lib().ftsp_profile_read(self.h, None, 0, C.byref(n)), "profile_read")
        buf = (ftsp_kernel_stat * max(1, n.value))()
        self._check(lib().ftsp_profile_read(self.h, buf, n.value, C.byref(n)), "profile_read")
        return {buf[i].name.decode(): {"ms": buf[i].ms, "launches": buf[i].launches, "bytes": buf[i].bytes}
                for i in range(n.value)}

    def set_noise(self, eta):
        e = np.ascontiguousarray(np.asarray(eta, dtype=np.float64).reshape(-1))
        if e.size != (self.n_modes + 1) * self.size:
            raise ValueError("noise must hold (n_modes + 1) * V values")
        self._check(lib().ftsp_set_noise(self.h, e.ctypes.data), "set_noise")

    def step(self, eta=None):
        """One step; returns (Q_bar, record, drift_max)."""
        if eta is not None:
            self.set_noise(eta)
        Qb = np.zeros(max(1, self.n_species), dtype=np.complex128)
        rec = np.zeros(max(1, self.record_len), dtype=np.complex128)
        dmax = np.zeros(self.n_modes + 1)
        self._check(lib().ftsp_step(self.h, Qb.ctypes.data, rec.ctypes.data, dmax.ctypes.data), "step")
        return Qb[: self.n_species], rec[: self.record_len], dmax

    def step_async(self):
        self._check(lib().ftsp_step_async(self.h), "step_async")

    def read_status(self):
        rec = np.zeros(max(1, self.record_len), dtype=np.complex128)
        dmax = np.zeros(self.n_modes + 1)
        rc = lib().ftsp_read_status(self.h, rec.ctypes.data, dmax.ctypes.data)
        return rc, rec[: self.record_len], dmax

    def set_stream(self, stream_handle: int):
        self._check(lib().ftsp_set_stream(self.h, C.c_void_p(stream_handle)), "set_stream")

    def set_adaptive(self, u_ref: float):
        """Adaptive step: dt_eff = dt min(1, u_ref / max|u|); 0 switches it off."""
        self._check(lib().ftsp_set_adaptive(self.h, float(u_ref)), "set_adaptive")

    def set_chain_symmetry(self, on: bool) -> int:
        """Pair path for mirror-symmetric species (default on); returns how
        many species take it."""
        n = C.c_int()
        self._check(lib().ftsp_set_chain_symmetry(self.h, int(bool(on)), C.byref(n)), "set_chain_symmetry")
        return n.value

    def set_step_graph(self, on: bool):
        """Replay the step as a captured CUDA graph (default on)."""
        self._check(lib().ftsp_set_step_graph(self.h, int(bool(on))), "set_step_graph")

    def step_info(self):
        """(dt_eff, max|u|) of the last step."""
        a, b = C.c_double(), C.c_double()
        self._check(lib().ftsp_step_info(self.h, C.byref(a), C.byref(b)), "step_info")
        return a.value, b.value

    def tune_info(self) -> dict:
        t = ftsp_tune_info()
        self._check(lib().ftsp_tune_info_get(self.h, C.byref(t)), "tune_info")
        return {k: getattr(t, k) for k, _ in t._fields_}

    # ---- time step and learned preconditioner (include/ftsp.h) ----
    def set_dt(self, dt: float):
        self._check(lib().ftsp_set_dt(self.h, float(dt)), "set_dt")

    def learn_configure(self, N: float, lB: float, salt: float, lr: float = 1e-3, batch: int = 4096,
                        refresh_every: int = 100, fallback_ratio: float = 1.5, seed: int = 7):
        cf = ftsp_learn_config(float(N), float(lB), float(salt), float(lr), int(batch), int(refresh_every),
                               float(fallback_ratio), int(seed))
        self._check(lib().ftsp_learn_configure(self.h, C.byref(cf)), "learn_configure")

    def learn_collect(self, on: bool = True):
        self._check(lib().ftsp_learn_collect(self.h, int(bool(on))), "learn_collect")

    def learn_reset(self):
        self._check(lib().ftsp_learn_reset(self.h), "learn_reset")

    def learn_train(self, iterations: int) -> float:
        loss = C.c_double()
        self._check(lib().ftsp_learn_train(self.h, int(iterations), C.byref(loss)), "learn_train")
        return loss.value

    def learn_use(self, on: bool = True):
        self._check(lib().ftsp_learn_use(self.h, int(bool(on))), "learn_use")

    def learn_stats(self) -> dict:
        st = ftsp_learn_stats()
        self._check(lib().ftsp_learn_get_stats(self.h, C.byref(st)), "learn_get_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def learn_weights(self) -> np.ndarray:
        n = C.c_int(0)
        self._check(lib().ftsp_learn_get_weights(self.h, None, C.byref(n)), "learn_get_weights")
        w = np.zeros(n.value, dtype=np.float32)
        self._check(lib().ftsp_learn_get_weights(self.h, w.ctypes.data, C.byref(n)), "learn_get_weights")
        return w

    def learn_set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(lib().ftsp_learn_set_weights(self.h, w.ctypes.data, int(w.size)), "learn_set_weights")

    def learn_grad(self, x: np.ndarray, t: np.ndarray, m: np.ndarray):
        """(loss, gradient) of the network on caller samples, through the GPU kernels."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        m = np.ascontiguousarray(m, dtype=np.float32)
        n = x.shape[0]
        g = np.zeros(self.learn_weights().size, dtype=np.float32)
        loss = C.c_double()
        self._check(lib().ftsp_learn_grad(self.h, x.ctypes.data, t.ctypes.data, m.ctypes.data, int(n), C.byref(loss),
                                          g.ctypes.data), "learn_grad")
        return loss.value, g

    def restarts(self) -> int:
        return int(lib().ftsp_restart_count(self.h))

    def average_start(self, skip: int, samples: int, blocks: int = 10):
        """Starts device-side time averaging of the record: steps after the
        first `skip`, at most `samples` finite records, in `blocks` blocks."""
        self._check(lib().ftsp_average_start(self.h, int(skip), int(samples), int(blocks)), "average_start")

    def average_read(self):
        """(mean, standard error, records accumulated): real parts of the
        record entries, the error from the block means."""
        mean = np.zeros(self.record_len)
        se = np.zeros(self.record_len)
        n = C.c_longlong()
        self._check(lib().ftsp_average_read(self.h, mean.ctypes.data, se.ctypes.data, C.byref(n)), "average_read")
        return mean, se, int(n.value)

    def rollback_exhausted(self) -> bool:
        """True once a non-finite step found max_restarts rollbacks already
        taken: the run is over (every later step is non-finite) until
        set_fields starts a new one."""
        r = C.c_longlong()
        x = C.c_int()
        self._check(lib().ftsp_rollback_info(self.h, C.byref(r), C.byref(x)), "rollback_info")
        return bool(x.value)

    def launches(self) -> int:
        return int(lib().ftsp_last_launch_count(self.h))

    def views(self) -> ftsp_views:
        v = ftsp_views()
        self._check(lib().ftsp_state_views(self.h, C.byref(v)), "state_views")
        return v


class Batch:
    """Independent replicas stepped together: `steps_per_graph` steps of every
    engine captured into one CUDA graph (one branch stream per engine), one
    graph launch per `step` call.  The engines must outlive the batch and are
    not stepped on their own while it exists."""

    def __init__(self, engines, steps_per_graph: int = 1):
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e.h.value for e in self.engines])
        h = C.c_void_p()
        if lib().ftsp_batch_create(arr, len(self.engines), int(steps_per_graph), C.byref(h)) != FTSP_OK:
            raise FtspError("ftsp_batch_create: " + (lib().ftsp_batch_last_error(None) or b"").decode())
        self.h = h
        self.steps_per_graph = int(steps_per_graph)
        self.launches_per_graph = int(lib().ftsp_batch_launch_count(self.h))

    def stream(self) -> int:
        return int(lib().ftsp_batch_stream(self.h) or 0)

    def step(self, graph_launches: int = 1):
        if lib().ftsp_batch_step(self.h, int(graph_launches)) != FTSP_OK:
            raise FtspError("ftsp_batch_step: " + (lib().ftsp_batch_last_error(self.h) or b"").decode())

    def sync(self):
        if lib().ftsp_batch_sync(self.h) != FTSP_OK:
            raise FtspError("ftsp_batch_sync: " + (lib().ftsp_batch_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            lib().ftsp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
