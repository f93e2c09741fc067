"""Parity on the named workloads, through the C ABI, against the FP64 oracle.

  * workload 4 (128^3, L = 64 b, N = 50, divalent counterions, salt 0.05,
    full stress + isotropic pressure) -- the benchmark configuration: one
    density evaluation and the observable record in complex128 and in
    complex64.  The uniform chain is mirror-symmetric, so the engine runs
    the benchmark's path: one forward sweep (complex64: the fused plane pass
    k_plane_fused and the fused bond pass k_strided_fused) and the pair
    density / pair stress kernels.  The oracle re-solves the chains for every
    stress component, as the reference does (stress.cu:161-196), so it is
    asked for sigma_xx, sigma_xy and the isotropic pressure only; the engine
    computes all six components and those three are compared.  Then one
    semi-implicit step in complex64 against the engine's complex128 step on
    the same fields and noise (the complex128 SI step itself is checked
    against the numpy restatement in test_gpu_si).
  * workload 1 (32^3, N = 32, complex128, the reference's predictor-corrector):
    one step at 1e-10, then a 200-step trajectory with the same injected
    noise in both, whose drift from the oracle is reported and bounded.
  * workload 2 (64^3, N = 50, complex64): one predictor-corrector step against
    the oracle, and one semi-implicit step against the engine's complex128 one.

Tolerances as elsewhere: complex128 1e-10 on fields (relative to the field's
largest modulus) and on records (relative, floor 1e-3); complex64 1e-5 on
fields and 2e-3 on records.
"""
import numpy as np
import pytest

import pyoracle as po
from ftspolysol_b200.cases import workload
from ftspolysol_b200.derive import derive

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(float(np.max(np.abs(b))), 1e-300))


def rec_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3)))


def record_names(d):
    """Labels of the record entries (observable.h:7-13 order)."""
    S, J = len(d["species"]), len(d["ions"])
    names = ["mu_ex_%d" % i for i in range(S + J)] + ["mu_self_%d" % i for i in range(S + J)]
    names += ["mu_id_%d" % i for i in range(S + J)] + ["H"]
    names += ["stress_" + c for c in d["stress"]]
    if d.get("isotropic_pressure"):
        names.append("Pi")
    return names


# --------------------------------------------------------------------------
# workload 4: the benchmark configuration
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def w4():
    case = workload(4, noise=False)
    d = derive(case)
    om, ps = case.initial_fields()
    d_or = dict(d, stress=("xx", "xy"))
    o = po.Oracle(d_or)
    o.set_fields(om, ps)
    Q = o.compute_densities(0)
    rho = o.get("rho_type")
    rho_c = o.get("rho_c")
    ion_rho = o.get("ion_rho")
    rec = o.measure(0, Q)
    o.close()
    return {"case": case, "d": d, "d_or": d_or, "om": om, "ps": ps, "Q": Q, "rho": rho, "rho_c": rho_c,
            "ion_rho": ion_rho, "rec": rec}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_workload4_densities_and_record(w4, prec):
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    ftol, rtol = (1e-10, 1e-10) if prec == "fp64" else (1e-5, 2e-3)
    eng = Engine(w4["d"], precision=FP64 if prec == "fp64" else FP32, scheme=SCHEME_SI)
    eng.set_fields(w4["om"], w4["ps"])
    assert rel(eng.compute_densities(0), w4["Q"]) < ftol
    assert rel(eng.get("rho_type"), w4["rho"]) < ftol
    assert rel(eng.get("rho_c"), w4["rho_c"]) < ftol
    assert rel(eng.get("ion_rho"), w4["ion_rho"]) < ftol
    rec = eng.measure(0)
    eng.close()
    full = record_names(w4["d"])
    sub = record_names(w4["d_or"])
    ours = np.array([rec[full.index(n)] for n in sub])
    assert rec_err(ours, w4["rec"]) < rtol, dict(zip(sub, np.abs(ours - w4["rec"]) / np.maximum(np.abs(w4["rec"]), 1e-3)))


def test_workload4_fp32_si_step_matches_fp64(w4):
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    case = w4["case"]
    eta = np.random.default_rng(23).standard_normal((2, case.size)) * np.sqrt(2 * 0.005 / 0.125)
    out = {}
    for prec in (FP64, FP32):
        eng = Engine(w4["d"], precision=prec, scheme=SCHEME_SI)
        eng.set_fields(w4["om"], w4["ps"])
        Q, rec, _ = eng.step(eta)
        out[prec] = (Q, rec, eng.get("omega"), eng.get("psi"), eng.get("rho_type"))
        eng.close()
    a, b = out[FP64], out[FP32]
    assert rel(b[0], a[0]) < 1e-5
    assert rec_err(b[1], a[1]) < 2e-3
    for x, y in zip(b[2:], a[2:]):
        assert rel(x, y) < 1e-5


# --------------------------------------------------------------------------
# workload 1: 32^3 FP64, the reference scheme; one step and a trajectory
# --------------------------------------------------------------------------
def test_workload1_step_and_trajectory():
    from ftspolysol_b200 import Engine, FP64, SCHEME_PC
    case = workload(1, noise=False)
    d = derive(case)
    om, ps = case.initial_fields()
    sigma = np.sqrt(2.0 * 1.0 * d["dt"] / d["dV"])   # lambda = 1 (complexLangevin.cu:287-297)
    rng = np.random.default_rng(41)
    o = po.Oracle(d)
    o.set_fields(om, ps)
    eng = Engine(d, precision=FP64, scheme=SCHEME_PC)
    eng.set_fields(om, ps)
    drift = []
    for k in range(200):
        eta = rng.standard_normal((2, case.size)) * sigma
        Qo, reco, _ = o.step(eta)
        Qe, rece, _ = eng.step(eta)
        if k == 0:   # single-step parity
            assert rel(Qe, Qo) < 1e-10
            assert rec_err(rece, reco) < 1e-10
            assert rel(eng.get("omega"), o.get("omega")) < 1e-10
            assert rel(eng.get("psi"), o.get("psi")) < 1e-10
        if (k + 1) % 50 == 0:
            drift.append((k + 1, rel(eng.get("omega"), o.get("omega")), rel(eng.get("psi"), o.get("psi")),
                          rec_err(rece, reco)))
    o.close()
    eng.close()
    print("workload 1 trajectory drift (step, omega, psi, record):", drift)
    # rounding differences (own FFT vs the oracle's) grow along the
    # trajectory but stay far below the statistical noise of the run
    for _, dw, dp, dr in drift:
        assert np.isfinite(dw) and dw < 1e-6
        assert np.isfinite(dp) and dp < 1e-6
        assert dr < 1e-6


# --------------------------------------------------------------------------
# workload 2: 64^3 complex64
# --------------------------------------------------------------------------
def test_workload2_fp32_step():
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_PC, SCHEME_SI
    case = workload(2, noise=False)
    d = derive(case)
    om, ps = case.initial_fields()
    eta = np.random.default_rng(29).standard_normal((2, case.size)) * np.sqrt(2 * d["dt"] / d["dV"])
    o = po.Oracle(d)
    o.set_fields(om, ps)
    Qo, reco, _ = o.step(eta)
    om1, ps1 = o.get("omega"), o.get("psi")
    o.close()
    e = Engine(d, precision=FP32, scheme=SCHEME_PC)
    e.set_fields(om, ps)
    Q, rec, _ = e.step(eta)
    assert rel(Q, Qo) < 1e-5
    assert rec_err(rec, reco) < 2e-3
    assert rel(e.get("omega"), om1) < 1e-5
    assert rel(e.get("psi"), ps1) < 1e-5
    e.close()
    out = {}
    for prec in (FP64, FP32):
        e = Engine(d, precision=prec, scheme=SCHEME_SI)
        e.set_fields(om, ps)
        Q, rec, _ = e.step(eta)
        out[prec] = (Q, rec, e.get("omega"), e.get("psi"))
        e.close()
    assert rel(out[FP32][0], out[FP64][0]) < 1e-5
    assert rec_err(out[FP32][1], out[FP64][1]) < 2e-3
    assert rel(out[FP32][2], out[FP64][2]) < 1e-5
    assert rel(out[FP32][3], out[FP64][3]) < 1e-5
