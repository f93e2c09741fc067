"""Derived parameters of a Case (what the reference's setup computes).

Restates, for cases built in Python: param::derive and
recompute_polymer_derived (param.cu:342-359, 412-436), the interaction-mode
decomposition (interactionMode.cu:9-59, 214-263: K_ab = xi + chi_ab with
K_aa = xi, eigenpairs sorted by decreasing eigenvalue, each eigenvector's
largest-magnitude component made positive, modes with |d| above
eigen_tol_rel * max(1, max|d|) active, gamma = i for d > 0 else 1), the
mobility list (param.cu:387-410), ion::build (ion.cu:3-46, counterion
auto-neutralisation, salt stoichiometry, merging of identical species) and
param::short_range_self_pressure (param.cu:130-147).
"""
from __future__ import annotations

import math

import numpy as np

from .cases import Case


def _jacobi(K: np.ndarray):
    """Cyclic Jacobi eigen-decomposition of a real symmetric matrix, with the
    sweep order, rotation formulas and convergence test of the reference's
    interactionMode::jacobi_symmetric_eigen (interactionMode.cu:122-194), so
    that eigenvector signs, and the pivot of degenerate |components|, come
    out as in the reference (numpy's eigh may differ in the last bit)."""
    n = K.shape[0]
    a = [[float(K[i, j]) for j in range(n)] for i in range(n)]
    v = [[1.0 if i == j else 0.0 for j in range(n)] for i in range(n)]
    if n == 1:
        return np.array([a[0][0]]), np.array(v)

    def frob(m):
        return math.sqrt(sum(x * x for row in m for x in row))

    def off(m):
        return math.sqrt(sum(m[i][j] * m[i][j] for i in range(n) for j in range(n) if i != j))

    scale = max(1.0, frob(a))
    tol = 1e-14 * scale
    eps = np.finfo(float).eps
    for _ in range(max(50, 100 * n * n)):
        if off(a) <= tol:
            break
        rotated = False
        for p in range(n - 1):
            for q in range(p + 1, n):
                apq = a[p][q]
                if abs(apq) <= eps * scale:
                    continue
                app, aqq = a[p][p], a[q][q]
                tau = (aqq - app) / (2.0 * apq)
                t = 1.0 / (tau + math.sqrt(1.0 + tau * tau)) if tau >= 0.0 else -1.0 / (-tau + math.sqrt(1.0 + tau * tau))
                c = 1.0 / math.sqrt(1.0 + t * t)
                s = t * c
                for k in range(n):
                    if k == p or k == q:
                        continue
                    akp, akq = a[k][p], a[k][q]
                    nkp, nkq = c * akp - s * akq, s * akp + c * akq
                    a[k][p] = a[p][k] = nkp
                    a[k][q] = a[q][k] = nkq
                a[p][p] = c * c * app - 2.0 * s * c * apq + s * s * aqq
                a[q][q] = s * s * app + 2.0 * s * c * apq + c * c * aqq
                a[p][q] = a[q][p] = 0.0
                for k in range(n):
                    vkp, vkq = v[k][p], v[k][q]
                    v[k][p] = c * vkp - s * vkq
                    v[k][q] = s * vkp + c * vkq
                rotated = True
        if not rotated:
            break
    return np.array([a[i][i] for i in range(n)]), np.array(v)


def interaction_modes(M: int, xi: float, chi: np.ndarray, tol_rel: float):
    """Modes of K = xi + chi (diagonal xi): eigenvalues in descending order,
    eigenvectors as rows with the largest-|component| entry made positive
    (first index on ties), active modes above tol_rel * max(1, max|d|)
    (interactionMode.cu:196-263)."""
    K = xi + np.asarray(chi, dtype=np.float64).reshape(M, M)
    np.fill_diagonal(K, xi)
    d, vec = _jacobi(K)
    order = sorted(range(M), key=lambda i: (-d[i], i))
    evals = np.array([d[i] for i in order])
    O = np.array([vec[:, i] for i in order])   # row l = eigenvector of mode l
    for l in range(M):
        piv = 0
        for k in range(1, M):
            if abs(O[l, k]) > abs(O[l, piv]):
                piv = k
        if O[l, piv] < 0.0:
            O[l] *= -1.0
    tol = tol_rel * max(1.0, float(np.max(np.abs(evals))))
    active = [l for l in range(M) if abs(evals[l]) > tol]
    return K, evals, O, active


def build_ions(case: Case, polymer_charge: float):
    """ion::build: returns [(name, valence, count, smearing)]."""
    elec = case.lB > 0.0
    default_smear = case.default_smearing_length if case.default_smearing_length is not None else case.a
    out = []
    combine = True if case.salt is None else bool(case.salt.get("combine_identical_species", True))

    def append(name, z, count, smear):
        if count == 0:
            return
        if combine:
            for sp in out:
                if abs(sp[1] - z) <= 1e-12 and abs(sp[3] - smear) <= 1e-12:
                    sp[2] += count
                    return
        out.append([name, z, count, smear])

    if case.ions_enabled and case.counterions is not None:
        ci = case.counterions
        z = float(ci["valence"])
        num = ci.get("number", "auto_neutralize")
        if num == "auto_neutralize":
            if elec:
                need = -polymer_charge / z
                if need < -1e-10:
                    raise ValueError("invalid counterion sign")
                n = int(round(need))
                if abs(need - n) > 1e-8 * max(1.0, abs(need)):
                    raise ValueError("invalid counterion number")
            else:
                n = 0
        else:
            n = int(num)
        smear = ci.get("smearing_length") or default_smear
        append(ci.get("name", "counterion"), z, n, smear)
    if case.ions_enabled and case.salt is not None:
        s = case.salt
        smear = s.get("smearing_length") or default_smear
        ns = int(s["num_salt"])
        append(s.get("cation_name", "salt_cation"), float(s["cation_valence"]), ns * int(s.get("cation_stoich", 1)), smear)
        append(s.get("anion_name", "salt_anion"), float(s["anion_valence"]), ns * int(s.get("anion_stoich", 1)), smear)
    if elec:
        total = polymer_charge + sum(z * n for _, z, n, _ in out)
        scale = abs(polymer_charge) + sum(abs(z * n) for _, z, n, _ in out)
        if abs(total) > 1e-8 * max(1.0, scale):
            raise ValueError("electroneutrality failed")
    return out


def derive(case: Case) -> dict:
    m = tuple(int(v) for v in case.m)
    L = case.L
    V = L[0] * L[1] * L[2]
    M = case.M
    names = list(case.monomer_names)
    species = []
    total_segments = 0
    type_segments = [0] * M
    polymer_charge = 0.0
    for sp in case.species:
        N = sp.N
        types = [names.index(t) for t in sp.monomers]
        bonds = [1.0] * N
        if sp.bonds is not None:
            for s in range(N - 1):
                bonds[s] = float(sp.bonds[s])
        species.append({"num_chains": float(sp.num_chains), "types": types,
                        "charges": [float(q) for q in sp.charges], "bonds": bonds})
        total_segments += sp.num_chains * N
        for t in types:
            type_segments[t] += sp.num_chains
        polymer_charge += sp.num_chains * sum(sp.charges)
    rho0 = total_segments / V
    K, evals, O, active = interaction_modes(M, case.xi, case.chi_matrix(), case.eigen_tol_rel)
    lam_in = list(case.lambda_omega)
    if len(lam_in) == 1:
        lam = lam_in * len(active)
    elif len(lam_in) == len(active):
        lam = lam_in
    else:
        raise ValueError("lambda_omega length must be 1 or the number of active modes")
    modes = []
    for i, l in enumerate(active):
        d = float(evals[l])
        modes.append({"coeff": rho0 / abs(d), "lambda": float(lam[i]), "gamma": 1j if d > 0 else 1.0 + 0j,
                      "eig": d, "O": [float(v) for v in O[l]]})
    ions = [{"name": n, "valence": z, "count": float(c), "smear": s}
            for n, z, c, s in build_ions(case, polymer_charge)]
    self_p = 0.0
    if case.a > 0 and total_segments > 0:
        mean_diag = sum(type_segments[a] * K[a, a] for a in range(M)) / total_segments
        self_p = mean_diag / (16.0 * math.pi * math.sqrt(math.pi) * case.a ** 3)
    return {"m": m, "L": L, "dV": case.dL ** 3, "volume": V, "rho0": rho0, "a": case.a, "lB": case.lB,
            "dt": case.dt, "lambda_psi": case.lambda_psi, "self_pressure": self_p, "M": M,
            "modes": modes, "ions": ions, "species": species, "stress": list(case.stress),
            "isotropic_pressure": bool(case.isotropic_pressure), "noise": bool(case.noise)}
