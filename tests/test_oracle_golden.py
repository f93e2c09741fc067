"""The FP64 CPU oracle against the reference's own CUDA build.

The golden vectors in tests/golden/*.npz were dumped by oracle/ref_harness.cu
driving the reference's unmodified classes (tests/golden/make_golden.py).
They pin the oracle: densities, propagators, partition functions, every
observable of the record (mu, H, stress components, isotropic pressure), the
drift maxima and three full predictor-corrector steps with injected noise.
"""
import os

import numpy as np
import pytest

import pyoracle as po

CASES = ["pe_small", "copoly_m2", "neutral_m2", "mix_m3", "short_neutral"]
FIELD_TOL = 1e-12      # relative to the field's max modulus
RECORD_TOL = 1e-10     # relative, floor 1e-3 for values near zero


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def record_err(rec, golden_flat):
    g = golden_flat.reshape(-1, 2)
    g = g[:, 0] + 1j * g[:, 1]
    assert rec.shape == g.shape
    return float(np.max(np.abs(rec - g) / np.maximum(np.abs(g), 1e-3)))


@pytest.fixture(scope="module", params=CASES)
def case(request, golden_dir):
    g = np.load(os.path.join(golden_dir, request.param + ".npz"))
    o = po.Oracle(po.derived_from_golden(g))
    o.set_fields(g["input_omega"], g["input_psi"])
    return request.param, g, o


def test_fft_matches_numpy():
    rng = np.random.default_rng(0)
    for shape in [(12, 8, 16), (6, 9, 10), (7, 5, 3), (32, 4, 2)]:
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        assert rel(po.fft3d(x, -1), np.fft.fftn(x)) < 1e-14
        assert rel(po.fft3d(x, +1), np.fft.ifftn(x) * x.size) < 1e-14


def test_tables(case):
    name, g, o = case
    assert rel(o.get("k2"), g["k2"]) < 1e-15
    assert rel(o.get("Gamma"), g["Gamma"]) < 1e-15


def test_initial_densities_and_observables(case):
    name, g, o = case
    assert rel(o.get("psi"), g["init_psi"]) < FIELD_TOL
    Q = o.compute_densities(0)
    assert rel(Q, g["init_Q"]) < FIELD_TOL
    for f in ["rho_type", "rho_p", "rho_c", "rho_c_poly", "rho_c_ion", "ion_rho", "W_type_s", "psi_s"]:
        if "init_" + f in g.files and np.max(np.abs(g["init_" + f])) > 0:
            assert rel(o.get(f), g["init_" + f]) < 1e-12, f
    if "init_qF" in g.files:
        assert rel(o.get("qF"), g["init_qF"]) < FIELD_TOL
        assert rel(o.get("qB"), g["init_qB"]) < FIELD_TOL
    assert record_err(o.measure(0, Q), g["init_record"]) < RECORD_TOL


def test_three_steps_with_noise(case):
    name, g, o = case
    o.set_fields(g["input_omega"], g["input_psi"])
    for st in range(1, 4):
        Qb, rec, dmax = o.step(g["noise"][st - 1])
        assert rel(Qb, g["step%d_bar_Q" % st]) < FIELD_TOL
        assert rel(o.get("omega"), g["step%d_omega" % st]) < FIELD_TOL
        if np.max(np.abs(g["step%d_psi" % st])) > 0:
            assert rel(o.get("psi"), g["step%d_psi" % st]) < FIELD_TOL
        assert record_err(rec, g["step%d_record" % st]) < RECORD_TOL
        assert rel(dmax, g["step%d_drift_max" % st]) < FIELD_TOL
