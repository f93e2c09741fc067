"""Python view of the host front end (include/ftsp_host.h).

``Model`` loads a reference param file and its sequence file with the C++
readers inside libftsp.so (param.cu / polymer.cu / interactionMode.cu /
ion.cu rules) and hands out the engine configuration; ``run_main`` runs the
reference-style program (main.cu) in this process.  Loading a model and the
field-file functions need no GPU; ``run_main`` does.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from .engine import FTSP_OK, ftsp_config, lib as _engine_lib

HOST_SYMBOLS = ("ftsp_model_load", "ftsp_model_free", "ftsp_model_config", "ftsp_model_get_info", "ftsp_model_modes",
                "ftsp_model_read_fields", "ftsp_model_write_omega", "ftsp_model_write_fields", "ftsp_main")


class ftsp_model_info(C.Structure):
    _fields_ = [("m1", C.c_int), ("m2", C.c_int), ("m3", C.c_int), ("M", C.c_int), ("n_modes", C.c_int),
                ("n_species", C.c_int), ("n_ions", C.c_int), ("Nt", C.c_int), ("Nss", C.c_int), ("Ns", C.c_int),
                ("Ntmp", C.c_int), ("Nso", C.c_int), ("N_stat", C.c_int), ("max_nan_restarts", C.c_int),
                ("noise", C.c_int), ("legacy_ab", C.c_int), ("rho0", C.c_double), ("volume", C.c_double),
                ("self_pressure", C.c_double), ("eigen_tol_abs", C.c_double), ("total_segments", C.c_longlong)]


_bound = False


def lib():
    global _bound
    L = _engine_lib()
    if not _bound:
        vp = C.c_void_p
        L.ftsp_model_load.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(vp)]
        L.ftsp_model_free.argtypes = [vp]
        L.ftsp_model_free.restype = None
        L.ftsp_model_config.argtypes = [vp, C.POINTER(ftsp_config)]
        L.ftsp_model_get_info.argtypes = [vp, C.POINTER(ftsp_model_info)]
        L.ftsp_model_modes.argtypes = [vp, vp, vp]
        L.ftsp_model_read_fields.argtypes = [vp, C.c_char_p, C.c_char_p, vp, vp]
        L.ftsp_model_write_omega.argtypes = [vp, C.c_char_p, vp]
        L.ftsp_model_write_fields.argtypes = [vp, C.c_char_p, C.c_int, vp]
        L.ftsp_main.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
        _bound = True
    return L


class ModelError(RuntimeError):
    pass


def _err() -> str:
    return (lib().ftsp_last_error(None) or b"").decode()


def _enc(s: Optional[str]):
    return None if s is None else os.fsencode(s)


class Model:
    """A parsed and validated param + sequence pair (main.cu:16-27)."""

    def __init__(self, param_file: str, sequence_file: Optional[str] = None):
        h = C.c_void_p()
        if lib().ftsp_model_load(_enc(param_file), _enc(sequence_file), C.byref(h)) != FTSP_OK:
            raise ModelError(_err())
        self.h = h
        self.info = ftsp_model_info()
        lib().ftsp_model_get_info(self.h, C.byref(self.info))
        self.mesh = (self.info.m1, self.info.m2, self.info.m3)
        self.size = self.info.m1 * self.info.m2 * self.info.m3

    def close(self):
        if getattr(self, "h", None):
            lib().ftsp_model_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def config(self) -> ftsp_config:
        """Engine configuration; its arrays point into this model."""
        cfg = ftsp_config()
        if lib().ftsp_model_config(self.h, C.byref(cfg)) != FTSP_OK:
            raise ModelError(_err())
        cfg._model = self   # keep the arrays alive
        return cfg

    def modes(self):
        M = self.info.M
        eig = np.zeros(M)
        O = np.zeros((M, M))
        lib().ftsp_model_modes(self.h, eig.ctypes.data, O.ctypes.data)
        return eig, O

    def read_fields(self, omega_file: Optional[str] = None, psi_file: Optional[str] = None):
        om = np.zeros((self.info.n_modes, self.size), dtype=np.complex128)
        ps = np.zeros(self.size, dtype=np.complex128)
        if lib().ftsp_model_read_fields(self.h, _enc(omega_file), _enc(psi_file), om.ctypes.data, ps.ctypes.data) != FTSP_OK:
            raise ModelError(_err())
        return om, ps

    def write_omega(self, path: str, omega: np.ndarray):
        om = np.ascontiguousarray(omega, dtype=np.complex128)
        if lib().ftsp_model_write_omega(self.h, _enc(path), om.ctypes.data) != FTSP_OK:
            raise ModelError(_err())

    def write_fields(self, path: str, fields: np.ndarray):
        f = np.ascontiguousarray(fields, dtype=np.complex128).reshape(-1, self.size)
        if lib().ftsp_model_write_fields(self.h, _enc(path), f.shape[0], f.ctypes.data) != FTSP_OK:
            raise ModelError(_err())


def run_main(args: Sequence[str]) -> int:
    """Runs the reference-style program in this process (exit status)."""
    argv = [b"ftsp_main"] + [os.fsencode(a) for a in args]
    arr = (C.c_char_p * len(argv))(*argv)
    return int(lib().ftsp_main(len(argv), arr))
