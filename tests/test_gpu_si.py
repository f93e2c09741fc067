"""Semi-implicit update and device checkpoint rollback.

The semi-implicit (SI) scheme has no reference counterpart: its pieces are
checked against the plain FP64 numpy restatement in oracle/si_oracle.py.
  * the preconditioner 1/(1 + lambda dt G(k)) against a direct O(N^2) double
    sum of the discrete-Gaussian-chain correlation function;
  * one SI step: predictor omega_bar = omega + IFFT[P FFT(-lambda dt u + eta)]
    and corrector omega' = omega + IFFT[P FFT(-lambda dt (u + u_bar)/2 + eta)]
    (likewise psi, zero mode removed), rebuilt from the engine's own drifts;
  * with G = 0 (lambda = 0 for every field) SI equals the reference scheme.
Tolerance 1e-10 relative (FP64; 1e-12 on the tables), 1e-5 for complex64
(the restatement is fed the engine's complex64 drifts, so the difference is
the complex64 rounding of the update itself).  The production grids (32^3,
64^3, 128^3) run the compile-time kernels, including the fused x-pencil
preconditioner pass (forward x, P(k)/V, inverse x in registers).  The
rollback tests inject NaN noise from the host: the next step restores the
checkpoint, and after max_restarts rollbacks a further non-finite step is
final until new fields are set.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from si_oracle import si_step, si_tables

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.parametrize("name", ["pe_small", "copoly_m2", "neutral_m2"])
def test_si_preconditioner_and_step(name, golden_dir):
    from ftspolysol_b200 import Engine, SCHEME_SI
    g = np.load(os.path.join(golden_dir, name + ".npz"))
    d = po.derived_from_golden(g)
    m = d["m"]
    eng = Engine(d, scheme=SCHEME_SI)
    P = eng.get("si_precond").real.reshape(-1, *m)
    ref = si_tables(d)
    for f in range(len(ref)):
        assert rel(P[f], ref[f]) < 1e-12, f
    om0, ps0 = g["input_omega"], g["input_psi"]
    eta = g["noise"][0]
    eng.set_fields(om0, ps0)
    ps0 = eng.get("psi")[0]           # zero mode removed
    eng.step(eta)
    nm = len(d["modes"])
    u = eng.get("drift").reshape(nm, *m)
    ub = eng.get("drift_bar").reshape(nm, *m)
    dpsi = eng.get("dpsi")[0].reshape(m)
    dpsib = eng.get("dpsi_bar")[0].reshape(m)
    elec = d["lB"] > 0
    eps = eta[nm].reshape(m) - (eta[nm].mean() if elec else 0.0)

    def prec(x, Pf):
        return np.fft.ifftn(Pf * np.fft.fftn(x))

    om0 = np.asarray(om0).reshape(nm, *m)
    for a, md in enumerate(d["modes"]):
        lam = md["lambda"]
        pred = om0[a] + prec(-d["dt"] * lam * u[a] + eta[a].reshape(m), ref[a])
        assert rel(eng.get("omega_bar")[a].reshape(m), pred) < 1e-10
        corr = om0[a] + prec(-0.5 * d["dt"] * lam * (u[a] + ub[a]) + eta[a].reshape(m), ref[a])
        assert rel(eng.get("omega")[a].reshape(m), corr) < 1e-10
    if elec:
        ps0 = ps0.reshape(m)
        pb = ps0 + prec(-d["dt"] * d["lambda_psi"] * dpsi + eps, ref[nm])
        pb -= pb.mean()
        assert rel(eng.get("psi_bar")[0].reshape(m), pb) < 1e-10
        pn = ps0 + prec(-0.5 * d["dt"] * d["lambda_psi"] * (dpsi + dpsib) + eps, ref[nm])
        pn -= pn.mean()
        assert rel(eng.get("psi")[0].reshape(m), pn) < 1e-10
    eng.close()


def test_si_without_mobility_equals_reference_scheme(golden_dir):
    from ftspolysol_b200 import Engine, SCHEME_PC, SCHEME_SI
    g = np.load(os.path.join(golden_dir, "pe_small.npz"))
    d = po.derived_from_golden(g)
    d = dict(d)
    d["modes"] = [dict(md, **{"lambda": 0.0}) for md in d["modes"]]
    d["lambda_psi"] = 0.0
    out = []
    for scheme in (SCHEME_PC, SCHEME_SI):
        eng = Engine(d, scheme=scheme)
        eng.set_fields(g["input_omega"], g["input_psi"])
        Q, rec, _ = eng.step(g["noise"][0])
        out.append((Q, rec, eng.get("omega"), eng.get("psi")))
        eng.close()
    for x, y in zip(out[0], out[1]):
        assert rel(x, y) < 1e-12


def test_rollback_after_injected_nan(golden_dir):
    from ftspolysol_b200 import Engine
    g = np.load(os.path.join(golden_dir, "pe_small.npz"))
    d = po.derived_from_golden(g)
    eng = Engine(d, restart_interval=1)
    eng.set_fields(g["input_omega"], g["input_psi"])
    eng.step(g["noise"][0])
    good = eng.get("omega").copy()
    bad_eta = g["noise"][1].copy()
    bad_eta[0, 3] = np.nan                  # host-side fault injection
    eng.set_noise(bad_eta)
    eng.step_async()
    status, _, _ = eng.read_status()
    assert status == 1                      # the step reports the non-finite value
    eng.step_async()                        # restores the checkpoint first, then steps
    status, _, _ = eng.read_status()
    assert status == 0
    assert eng.restarts() == 1
    assert np.all(np.isfinite(eng.get("omega")))
    # the restored state was the checkpoint taken after the first step
    eng2 = Engine(d, restart_interval=1)
    eng2.set_fields(g["input_omega"], g["input_psi"])
    eng2.step(g["noise"][0])
    assert rel(eng2.get("omega"), good) < 1e-15
    eng.close()
    eng2.close()


def pe_case(m, N, seed=3, valence=2.0, salt=0.05):
    from ftspolysol_b200.cases import Case, homopolymer
    V = (m * 0.5) ** 3
    return Case(name="si_%d" % m, m=(m, m, m), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
                species=[homopolymer("P", int(round(0.5 * V / N)), N)],
                counterions={"number": "auto_neutralize", "valence": valence},
                salt={"num_salt": int(round(salt * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                dt=0.005, stress=("xx", "yy", "zz", "xy", "xz", "yz"), isotropic_pressure=True, init_seed=seed)


@pytest.mark.parametrize("m,N", [(32, 16), (64, 12), (128, 50)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_si_production_grids(m, N, prec):
    """The SI tables and one SI step on the compile-time kernels against the
    numpy restatement; 128^3 with N = 50 and divalent counterions is the
    benchmark workload (complex64: the fused x-pencil preconditioner pass)."""
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    from ftspolysol_b200.derive import derive
    case = pe_case(m, N)
    d = derive(case)
    mm = tuple(d["m"])
    nm = len(d["modes"])
    ref = si_tables(d)
    eng = Engine(d, precision=FP64 if prec == "fp64" else FP32, scheme=SCHEME_SI)
    ttol, ftol = (1e-12, 1e-10) if prec == "fp64" else (1e-6, 1e-5)
    P = eng.get("si_precond").real.reshape(-1, *mm)
    for f in range(len(ref)):
        assert rel(P[f], ref[f]) < ttol, (f, rel(P[f], ref[f]))
    om, ps = case.initial_fields()
    eta = np.random.default_rng(17).standard_normal((nm + 1, case.size)) * 0.2
    eng.set_fields(om, ps)
    om0 = eng.get("omega").reshape(nm, *mm)
    ps0 = eng.get("psi")[0].reshape(mm)
    eng.step(eta)
    u = eng.get("drift").reshape(nm, *mm)
    ub = eng.get("drift_bar").reshape(nm, *mm)
    dp = eng.get("dpsi")[0].reshape(mm)
    dpb = eng.get("dpsi_bar")[0].reshape(mm)
    ob, pb, on, pn = si_step(d, ref, om0, ps0, u, ub, dp, dpb, eta)
    assert rel(eng.get("omega_bar").reshape(nm, *mm), ob) < ftol
    assert rel(eng.get("psi_bar")[0].reshape(mm), pb) < ftol
    assert rel(eng.get("omega").reshape(nm, *mm), on) < ftol
    assert rel(eng.get("psi")[0].reshape(mm), pn) < ftol
    eng.close()


def test_rollback_cap_makes_the_failure_final(golden_dir):
    """max_restarts = 2: two non-finite steps are rolled back; the third is
    final (no restore, every later step non-finite) until set_fields."""
    from ftspolysol_b200 import Engine
    g = np.load(os.path.join(golden_dir, "pe_small.npz"))
    d = po.derived_from_golden(g)
    eng = Engine(d, restart_interval=1, max_restarts=2)
    eng.set_fields(g["input_omega"], g["input_psi"])
    eng.step(g["noise"][0])
    bad_eta = g["noise"][1].copy()
    bad_eta[0, 3] = np.nan                  # host-side fault injection
    for k in range(3):
        eng.set_noise(bad_eta)
        eng.step_async()
        status, _, _ = eng.read_status()
        assert status == 1
        assert eng.restarts() == k          # the step first rolled back the previous failure
    assert not eng.rollback_exhausted()
    eng.step_async()                        # finds 2 rollbacks taken: final
    status, _, _ = eng.read_status()
    assert status == 1 and eng.restarts() == 2 and eng.rollback_exhausted()
    for _ in range(2):                      # good noise no longer helps
        eng.step_async()
        status, _, _ = eng.read_status()
        assert status == 1
    eng.set_fields(g["input_omega"], g["input_psi"])   # a new run
    assert not eng.rollback_exhausted() and eng.restarts() == 0
    eng.step(g["noise"][0])
    assert np.all(np.isfinite(eng.get("omega")))
    eng.close()
