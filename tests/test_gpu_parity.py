"""CUDA engine (FP64) against the oracle and the reference's golden dumps.

Everything goes through the C ABI (libftsp.so).  Tolerances: fields and
partition functions 1e-10 relative to the field's max modulus; observable
records 1e-10 relative with a 1e-3 floor for values near zero.
"""
import os

import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu

CASES = ["pe_small", "copoly_m2", "neutral_m2", "mix_m3", "short_neutral"]
FIELD_TOL = 1e-10
RECORD_TOL = 1e-10


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def record_err(rec, g):
    if g.dtype != np.complex128:
        g = g.reshape(-1, 2)
        g = g[:, 0] + 1j * g[:, 1]
    return float(np.max(np.abs(rec - g) / np.maximum(np.abs(g), 1e-3)))


@pytest.fixture(scope="module", params=CASES)
def case(request, golden_dir):
    from ftspolysol_b200 import Engine
    g = np.load(os.path.join(golden_dir, request.param + ".npz"))
    d = po.derived_from_golden(g)
    eng = Engine(d)
    yield request.param, g, d, eng
    eng.close()


def test_initial_densities(case):
    name, g, d, eng = case
    eng.set_fields(g["input_omega"], g["input_psi"])
    assert rel(eng.get("psi"), g["init_psi"]) < FIELD_TOL
    Q = eng.compute_densities(0)
    assert rel(Q, g["init_Q"]) < FIELD_TOL
    for f in ["rho_type", "rho_p", "rho_c", "rho_c_poly", "rho_c_ion", "ion_rho", "W_type_s", "psi_s"]:
        key = "init_" + f
        if key in g.files and np.max(np.abs(g[key])) > 0:
            assert rel(eng.get(f), g[key]) < FIELD_TOL, f
    if "init_qF" in g.files:
        assert rel(eng.get("qF"), g["init_qF"]) < FIELD_TOL


def test_initial_record(case):
    name, g, d, eng = case
    eng.set_fields(g["input_omega"], g["input_psi"])
    rec = eng.measure(0)
    assert record_err(rec, g["init_record"]) < RECORD_TOL


def test_three_steps_match_reference(case):
    name, g, d, eng = case
    eng.set_fields(g["input_omega"], g["input_psi"])
    for st in range(1, 4):
        Qb, rec, dmax = eng.step(g["noise"][st - 1])
        assert rel(Qb, g["step%d_bar_Q" % st]) < FIELD_TOL
        assert rel(eng.get("omega"), g["step%d_omega" % st]) < FIELD_TOL
        if np.max(np.abs(g["step%d_psi" % st])) > 0:
            assert rel(eng.get("psi"), g["step%d_psi" % st]) < FIELD_TOL
            assert rel(eng.get("dpsi_bar"), g["step%d_dpsi_bar" % st]) < FIELD_TOL
        assert rel(eng.get("omega_bar"), g["step%d_omega_bar" % st]) < FIELD_TOL
        assert record_err(rec, g["step%d_record" % st]) < RECORD_TOL
        assert rel(dmax, g["step%d_drift_max" % st]) < FIELD_TOL
