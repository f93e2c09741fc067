"""ctypes front end of the FP64 CPU oracle (oracle/libftsp_oracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py use it as the checker.  The product never imports
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libftsp_oracle.so")

STRESS_NAMES = ("xx", "yy", "zz", "xy", "xz", "yz")


class _Config(C.Structure):
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
    ]


def build(quiet: bool = True) -> str:
    """Compiles the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-C", HERE, "-s"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(_Config)]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_threads.restype = C.c_int
        L.oracle_set_fields.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_compute_densities.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_measure.restype = C.c_int
        L.oracle_measure.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_step.restype = C.c_int
        L.oracle_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_get.restype = C.c_longlong
        L.oracle_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        L.oracle_fft3d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Oracle:
    """One oracle system.  `derived` is a dict of the derived parameters:

    m (3 ints), L (3), dV, a, lB, dt, lambda_psi, M, modes (list of dicts with
    coeff, lambda, gamma (complex), O (M floats)), species (list of dicts with
    num_chains, types, charges, bonds (N floats; last unused)), ions (list of
    dicts with valence, count, smear), self_pressure, stress (component names),
    isotropic_pressure.
    """

    def __init__(self, derived: dict):
        self.d = derived
        m = derived["m"]
        self.m = tuple(int(v) for v in m)
        self.size = int(np.prod(self.m))
        modes = derived["modes"]
        self.n_modes = len(modes)
        self.M = int(derived["M"])
        self._keep = []

        def arr(x, dt=np.float64):
            a = np.ascontiguousarray(np.asarray(x, dtype=dt))
            if a.size == 0:
                a = np.zeros(1, dtype=dt)
            self._keep.append(a)
            return a

        cfg = _Config()
        cfg.m1, cfg.m2, cfg.m3 = self.m
        cfg.L1, cfg.L2, cfg.L3 = [float(v) for v in derived["L"]]
        cfg.dV = float(derived["dV"])
        cfg.a = float(derived["a"])
        cfg.lB = float(derived["lB"])
        cfg.dt = float(derived["dt"])
        cfg.lambda_psi = float(derived["lambda_psi"])
        cfg.M = self.M
        cfg.n_modes = self.n_modes
        cfg.mode_coeff = _dp(arr([md["coeff"] for md in modes]))
        g = []
        for md in modes:
            g += [complex(md["gamma"]).real, complex(md["gamma"]).imag]
        cfg.mode_gamma = _dp(arr(g))
        cfg.mode_O = _dp(arr([o for md in modes for o in md["O"]]))
        cfg.mode_lambda = _dp(arr([md["lambda"] for md in modes]))
        sp = derived["species"]
        self.n_species = len(sp)
        self.Ns = [len(s["types"]) for s in sp]
        cfg.n_species = len(sp)
        cfg.num_chains = _dp(arr([s["num_chains"] for s in sp]))
        cfg.N = _ip(arr(self.Ns, np.int32))
        cfg.seg_type = _ip(arr([t for s in sp for t in s["types"]], np.int32))
        cfg.seg_charge = _dp(arr([q for s in sp for q in s["charges"]]))
        cfg.seg_bond = _dp(arr([b for s in sp for b in s["bonds"]]))
        ions = derived["ions"]
        self.n_ions = len(ions)
        cfg.n_ions = len(ions)
        cfg.ion_valence = _dp(arr([i["valence"] for i in ions]))
        cfg.ion_count = _dp(arr([i["count"] for i in ions]))
        cfg.ion_smear = _dp(arr([i["smear"] for i in ions]))
        cfg.self_pressure = float(derived["self_pressure"])
        mask = 0
        for c in derived.get("stress", ()):
            mask |= 1 << STRESS_NAMES.index(c)
        cfg.stress_mask = mask
        cfg.isotropic_pressure = int(bool(derived.get("isotropic_pressure", False)))
        self.n_stress = bin(mask).count("1")
        self.record_len = 3 * (self.n_species + self.n_ions) + 1 + self.n_stress + cfg.isotropic_pressure
        self._cfg = cfg
        self.h = lib().oracle_create(C.byref(cfg))

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, omega, psi):
        o = np.ascontiguousarray(np.asarray(omega, dtype=np.complex128).reshape(self.n_modes, self.size))
        p = np.ascontiguousarray(np.asarray(psi, dtype=np.complex128).reshape(self.size))
        if o.size == 0:
            o = np.zeros(1, dtype=np.complex128)
        lib().oracle_set_fields(self.h, o.ctypes.data, p.ctypes.data)

    def compute_densities(self, which: int = 0) -> np.ndarray:
        Q = np.zeros(max(1, self.n_species), dtype=np.complex128)
        lib().oracle_compute_densities(self.h, which, Q.ctypes.data)
        return Q[: self.n_species]

    def measure(self, which: int, Q) -> np.ndarray:
        Qa = np.ascontiguousarray(np.asarray(Q, dtype=np.complex128))
        out = np.zeros(self.record_len + 1, dtype=np.complex128)
        k = lib().oracle_measure(self.h, which, Qa.ctypes.data, out.ctypes.data)
        return out[:k]

    def step(self, eta=None):
        Qb = np.zeros(max(1, self.n_species), dtype=np.complex128)
        rec = np.zeros(self.record_len + 1, dtype=np.complex128)
        dmax = np.zeros(self.n_modes + 1)
        if eta is not None:
            e = np.ascontiguousarray(np.asarray(eta, dtype=np.float64).reshape(-1))
            ptr = e.ctypes.data
        else:
            e = None
            ptr = None
        k = lib().oracle_step(self.h, ptr, Qb.ctypes.data, rec.ctypes.data, dmax.ctypes.data)
        return Qb[: self.n_species], rec[:k], dmax

    def get(self, name: str) -> np.ndarray:
        n = lib().oracle_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(max(1, n), dtype=np.float64)
        lib().oracle_get(self.h, name.encode(), out.ctypes.data)
        out = out[:n]
        if name in ("k2", "Gamma"):
            return out
        return out.view(np.complex128).reshape(-1, self.size)


def fft3d(data: np.ndarray, sign: int = -1) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(data, dtype=np.complex128)).copy()
    m1, m2, m3 = a.shape
    lib().oracle_fft3d(m1, m2, m3, a.ctypes.data, sign)
    return a


def derived_from_golden(g) -> dict:
    """Derived parameters as the REFERENCE computed them (dumped by the
    harness), plus the stress selection read from the case's param text."""
    s = g["derived_scalars"]
    m = (int(s[0]), int(s[1]), int(s[2]))
    M = int(s[14])
    nm = int(s[15])
    md = g["derived_modes"]
    per = 5 + M
    modes = []
    for a in range(nm):
        r = md[a * per:(a + 1) * per]
        modes.append({"coeff": r[0], "lambda": r[1], "gamma": complex(r[2], r[3]), "eig": r[4], "O": list(r[5:5 + M])})
    ions = []
    di = g["derived_ions"]
    for j in range(len(di) // 3):
        ions.append({"valence": di[3 * j], "count": di[3 * j + 1], "smear": di[3 * j + 2]})
    species = []
    dp = g["derived_polymers"]
    k = 0
    while k < len(dp):
        nc, N = dp[k], int(dp[k + 1])
        k += 2
        seg = dp[k:k + 3 * N].reshape(N, 3)
        k += 3 * N
        species.append({"num_chains": nc, "types": [int(t) for t in seg[:, 0]],
                        "charges": list(seg[:, 1]), "bonds": list(seg[:, 2])})
    text = bytes(g["param_text"]).decode()
    stress = []
    iso = False
    for line in text.splitlines():
        line = line.strip()
        for c in STRESS_NAMES:
            if line.replace(" ", "") == "component_%s=true" % c:
                stress.append(c)
        if line.replace(" ", "") == "isotropic_pressure=true":
            iso = True
    return {"m": m, "L": (s[3], s[4], s[5]), "dV": s[6], "volume": s[7], "rho0": s[8], "a": s[9],
            "lB": s[10], "dt": s[11], "lambda_psi": s[12], "self_pressure": s[13], "M": M,
            "modes": modes, "ions": ions, "species": species, "stress": stress, "isotropic_pressure": iso}
