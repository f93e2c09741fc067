"""FP64 numpy restatement of the semi-implicit update (test infrastructure).

The semi-implicit (SI) scheme has no counterpart in the reference: FTSPolySol
integrates with the explicit Euler-Maruyama predictor-corrector of
complexLangevin.cu:328-368.  The engine's SI scheme preconditions every
increment of that predictor-corrector in k-space,

    P_f(k) = 1 / (1 + lambda_f dt G_f(k)),

with the homogeneous-state linear response G of each Langevin field f:

    modes:  G_a(k) = c_a - Re(gamma_a^2) Gamma(k)^2 S_oo(k)   (c_a = rho0/|d_a|, param.cu:115-118)
    psi:    G_psi(k) = k^2 / (4 pi lB) + Gamma(k)^2 S_zz(k) + sum_j n_j z_j^2 Gamma_j(k)^2 / V

where Gamma(k) = exp(-a^2 k^2 / 2) is the bead smearing (common.h:290-293),
and S_ww(k) = sum over species of (n/V) sum_{s,t} w_s w_t prod_{bonds between
s and t} Phi_b(k) is the discrete-Gaussian-chain correlation of the segment
weights w (O_{a, type} for a mode, the valence for psi), Phi_b(k) =
exp(-b^2 k^2 / 6) (common.h:295-298).  G is clipped at zero; the zero mode
keeps c_a (modes) and 0 (psi).

Only the tests import this module; it is the checker of the engine's SI
tables and update, never part of the product path.
"""
from __future__ import annotations

import numpy as np


def k2_grid(m, L):
    k = [2 * np.pi * np.fft.fftfreq(mi, d=Li / mi) for mi, Li in zip(m, L)]
    return k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2


def chain_corr(k2, weights, bonds):
    """sum_{s,t} w_s w_t prod_{bonds between s and t} exp(-b^2 k^2 / 6).

    With one bond length b along the whole chain the product is phi^|s-t|
    (phi = exp(-b^2 k^2/6)), so S = c_0 + 2 sum_{d>=1} c_d phi^d with the
    scalar lag sums c_d = sum_s w_s w_{s+d}, evaluated by Horner's rule
    (O(N) grid passes).  Otherwise the direct O(N^2) double sum."""
    w = np.asarray(weights, dtype=np.float64)
    N = len(w)
    b = np.asarray(bonds[: max(0, N - 1)], dtype=np.float64)
    if N == 1:
        return np.full_like(k2, w[0] * w[0])
    if np.all(b == b[0]):
        c = np.array([np.dot(w[: N - d], w[d:]) for d in range(N)])
        phi = np.exp(-b[0] ** 2 * k2 / 6.0)
        acc = np.full_like(k2, c[N - 1])
        for d in range(N - 2, 0, -1):
            acc = c[d] + phi * acc
        return c[0] + 2.0 * phi * acc
    S = np.zeros_like(k2)
    for s in range(N):
        prod = np.ones_like(k2)
        S += w[s] * w[s]
        for t in range(s + 1, N):
            prod = prod * np.exp(-b[t - 1] ** 2 * k2 / 6.0)
            S += 2.0 * w[s] * w[t] * prod
    return S


def si_tables(d):
    """P_f(k) for every Langevin field of the derived parameters d (modes, then psi)."""
    m = d["m"]
    k2 = k2_grid(m, d["L"])
    G2 = np.exp(-d["a"] ** 2 * k2)
    V = d["volume"]
    out = []
    for md in d["modes"]:
        S = np.zeros_like(k2)
        for sp in d["species"]:
            o = [md["O"][t] for t in sp["types"]]
            S += sp["num_chains"] / V * chain_corr(k2, o, sp["bonds"])
        g2 = (complex(md["gamma"]) ** 2).real
        G = md["coeff"] - g2 * G2 * S
        G[0, 0, 0] = md["coeff"]
        G = np.maximum(G, 0.0)
        out.append(1.0 / (1.0 + d["dt"] * md["lambda"] * G))
    Gp = np.zeros_like(k2)
    if d["lB"] > 0:
        S = np.zeros_like(k2)
        for sp in d["species"]:
            S += sp["num_chains"] / V * chain_corr(k2, sp["charges"], sp["bonds"])
        Gp = k2 / (4 * np.pi * d["lB"]) + G2 * S
        for ion in d["ions"]:
            Gp = Gp + ion["count"] / V * ion["valence"] ** 2 * np.exp(-ion["smear"] ** 2 * k2)
        Gp[0, 0, 0] = 0.0
    out.append(1.0 / (1.0 + d["dt"] * d["lambda_psi"] * Gp))
    return out


def si_step(d, P, omega0, psi0, u, ub, dpsi, dpsib, eta):
    """One SI predictor-corrector step rebuilt from the drifts the engine
    evaluated (u, ub at omega and omega_bar; dpsi, dpsib the raw psi drifts
    before their mean removal is applied by the update):

        omega_bar = omega + IFFT[P FFT(-lambda dt u + eta)]
        omega'    = omega + IFFT[P FFT(-lambda dt (u + u_bar)/2 + eta)]

    and likewise psi with lambda_psi, the psi noise and drifts with their
    means removed, and the zero mode of the result removed
    (complexLangevin.cu:313-368).  Arrays are shaped (fields, *m); returns
    (omega_bar, psi_bar, omega', psi')."""
    m = tuple(d["m"])
    nm = len(d["modes"])
    dt = d["dt"]
    elec = d["lB"] > 0

    def prec(x, Pf):
        return np.fft.ifftn(Pf * np.fft.fftn(x))

    ob, on = [], []
    for a, md in enumerate(d["modes"]):
        lam = md["lambda"]
        ob.append(omega0[a] + prec(-dt * lam * u[a] + eta[a].reshape(m), P[a]))
        on.append(omega0[a] + prec(-0.5 * dt * lam * (u[a] + ub[a]) + eta[a].reshape(m), P[a]))
    pb = pn = np.zeros(m, dtype=np.complex128)
    if elec:
        eps = eta[nm].reshape(m) - eta[nm].mean()
        lp = d["lambda_psi"]
        dp = dpsi - dpsi.mean()
        dpb = dpsib - dpsib.mean()
        pb = psi0 + prec(-dt * lp * dp + eps, P[nm])
        pb = pb - pb.mean()
        pn = psi0 + prec(-0.5 * dt * lp * (dp + dpb) + eps, P[nm])
        pn = pn - pn.mean()
    return np.array(ob), pb, np.array(on), pn
