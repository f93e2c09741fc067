"""Semi-implicit update and device checkpoint rollback.

The semi-implicit (SI) scheme has no reference counterpart: its pieces are
checked against plain FP64 numpy restatements.
  * the preconditioner 1/(1 + lambda dt G(k)) against a direct O(N^2) double
    sum of the discrete-Gaussian-chain correlation function;
  * one SI step: predictor omega_bar = omega + IFFT[P FFT(-lambda dt u + eta)]
    and corrector omega' = omega + IFFT[P FFT(-lambda dt (u + u_bar)/2 + eta)]
    (likewise psi, zero mode removed), rebuilt from the engine's own drifts;
  * with G = 0 (lambda = 0 for every field) SI equals the reference scheme.
Tolerance 1e-10 relative (FP64).  The rollback test injects NaN noise from
the host and checks that the next step restores the checkpoint.
"""
import os

import numpy as np
import pytest

import pyoracle as po

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(float(np.max(np.abs(b))), 1e-300))


def k2_grid(m, L):
    k = [2 * np.pi * np.fft.fftfreq(mi, d=Li / mi) for mi, Li in zip(m, L)]
    return k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2


def si_tables(d):
    m = d["m"]
    k2 = k2_grid(m, d["L"])
    G2 = np.exp(-d["a"] ** 2 * k2)
    V = d["volume"]
    out = []

    def corr(weights, bonds, N):
        S = np.zeros_like(k2)
        for s in range(N):
            prod = np.ones_like(k2)
            S += weights[s] * weights[s]
            for t in range(s + 1, N):
                prod = prod * np.exp(-bonds[t - 1] ** 2 * k2 / 6.0)
                S += 2.0 * weights[s] * weights[t] * prod
        return S

    for md in d["modes"]:
        S = np.zeros_like(k2)
        for sp in d["species"]:
            o = [md["O"][t] for t in sp["types"]]
            S += sp["num_chains"] / V * corr(o, sp["bonds"], len(o))
        g2 = (complex(md["gamma"]) ** 2).real
        G = md["coeff"] - g2 * G2 * S
        G[0, 0, 0] = md["coeff"]
        G = np.maximum(G, 0.0)
        out.append(1.0 / (1.0 + d["dt"] * md["lambda"] * G))
    Gp = np.zeros_like(k2)
    if d["lB"] > 0:
        S = np.zeros_like(k2)
        for sp in d["species"]:
            S += sp["num_chains"] / V * corr(sp["charges"], sp["bonds"], len(sp["charges"]))
        Gp = k2 / (4 * np.pi * d["lB"]) + G2 * S
        for ion in d["ions"]:
            Gp = Gp + ion["count"] / V * ion["valence"] ** 2 * np.exp(-ion["smear"] ** 2 * k2)
        Gp[0, 0, 0] = 0.0
    out.append(1.0 / (1.0 + d["dt"] * d["lambda_psi"] * Gp))
    return out


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
