"""Mirror-symmetric chains: densities and connectivity stress from the
forward sweep alone (pair kernels) against the oracle (which runs both
sweeps) and against the engine's own two-sweep path on the same inputs.

Cases: charged homopolymer (one class, one bond class), an ABA triblock
with an odd number of segments (middle segment pairs with itself), charged
ends and mirror-symmetric bond lengths (several bond classes), and a system
with a symmetric ABBA chain beside an asymmetric diblock (only the first
takes the pair path).  Grids cover the runtime-plan passes (odd extents,
Nyquist planes in every direction) and the 32^3 compile-time passes.
FP64 tolerances as for the other oracle tests (1e-10); the two engine paths
agree to 1e-12 in FP64 and 1e-5 / 2e-4 (fields / records) in complex64.
"""
import numpy as np
import pytest

import pyoracle as po
from ftspolysol_b200.cases import Case, Species, homopolymer
from ftspolysol_b200.derive import derive

pytestmark = pytest.mark.gpu

STRESS = ("xx", "yy", "zz", "xy", "xz", "yz")


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(float(np.max(np.abs(b))), 1e-300))


def rec_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3)))


def homo_case(m, N):
    V = (m[0] * 0.5) * (m[1] * 0.5) * (m[2] * 0.5)
    return Case(name="sym_homo", m=m, dL=0.5, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
                species=[homopolymer("P", max(2, int(round(0.4 * V / N))), N)],
                counterions={"number": "auto_neutralize", "valence": 1.0},
                salt={"num_salt": int(round(0.05 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                dt=0.01, stress=STRESS, isotropic_pressure=True, init_seed=5)


def triblock_case(m):
    # A3 B3 A3, charged A ends, bonds mirror-symmetric with four lengths
    mons = ["A"] * 3 + ["B"] * 3 + ["A"] * 3
    ch = [-1.0] * 3 + [0.0] * 3 + [-1.0] * 3
    bonds = [1.0, 0.9, 1.2, 0.8, 0.8, 1.2, 0.9, 1.0]
    V = (m[0] * 0.5) * (m[1] * 0.5) * (m[2] * 0.5)
    return Case(name="sym_aba", m=m, dL=0.5, monomer_names=["A", "B"], chi=[0.0, 0.6, 0.6, 0.0], xi=0.2, lB=1.0,
                species=[Species("T", max(2, int(round(0.3 * V / 9))), mons, ch, bonds)],
                counterions={"number": "auto_neutralize", "valence": 1.0},
                dt=0.01, stress=STRESS, isotropic_pressure=True, init_seed=7)


def mixed_case(m):
    # symmetric A B B A (even N: the middle bond pairs with itself) beside an asymmetric A A B B B
    abba = Species("S", 6, ["A", "B", "B", "A"], [1.0, 0.0, 0.0, 1.0], [0.9, 1.1, 0.9])
    diblock = Species("D", 6, ["A", "A", "B", "B", "B"], [-1.0, -1.0, 0.0, 0.0, 0.0])
    return Case(name="sym_mixed", m=m, dL=0.5, monomer_names=["A", "B"], chi=[0.0, 0.4, 0.4, 0.0], xi=0.15,
                lB=0.7, species=[abba, diblock], counterions=None,
                salt={"num_salt": 4, "cation_valence": 1.0, "anion_valence": -1.0},
                dt=0.01, stress=STRESS, isotropic_pressure=True, init_seed=9)


CASES = [(homo_case, (10, 12, 9), 7, 1), (homo_case, (16, 8, 12), 8, 1), (triblock_case, (12, 10, 8), None, 1),
         (mixed_case, (10, 8, 12), None, 1)]


def build(fn, m, N):
    return fn(m, N) if N is not None else fn(m)


@pytest.mark.parametrize("fn,m,N,nsym", CASES)
def test_pair_path_matches_oracle_and_two_sweeps(fn, m, N, nsym):
    from ftspolysol_b200 import Engine, FP64
    case = build(fn, m, N)
    d = derive(case)
    om, ps = case.initial_fields()
    eta = np.random.default_rng(3).standard_normal((len(d["modes"]) + 1, case.size)) * 0.2
    o = po.Oracle(d)
    o.set_fields(om, ps)
    Q0 = o.compute_densities(0)
    rho0 = o.get("rho_type")
    rec0 = o.measure(0, Q0)
    o.set_fields(om, ps)
    Qb, recb, _ = o.step(eta)
    omega1 = o.get("omega")
    o.close()
    res = []
    for on in (True, False):
        eng = Engine(d, precision=FP64)
        n = eng.set_chain_symmetry(on)
        assert n == (nsym if on else 0)
        eng.set_fields(om, ps)
        Q = eng.compute_densities(0)
        r = {"Q": Q, "rho": eng.get("rho_type"), "rho_c": eng.get("rho_c"), "qF": eng.get("qF"),
             "rec": eng.measure(0)}
        eng.set_fields(om, ps)
        Qs, rec, _ = eng.step(eta)
        r.update(Qs=Qs, rec1=rec, omega=eng.get("omega"), psi=eng.get("psi"))
        eng.close()
        assert rel(r["Q"], Q0) < 1e-10
        assert rel(r["rho"], rho0) < 1e-10
        assert rec_err(r["rec"], rec0) < 1e-10
        assert rel(r["Qs"], Qb) < 1e-10
        assert rec_err(r["rec1"], recb) < 1e-10
        assert rel(r["omega"], omega1) < 1e-10
        res.append(r)
    a, b = res
    for k in ("rho", "rho_c", "qF", "omega", "psi"):
        if np.max(np.abs(b[k])) > 0:
            assert rel(a[k], b[k]) < 1e-12, k
    assert rec_err(a["rec"], b["rec"]) < 1e-11
    assert rec_err(a["rec1"], b["rec1"]) < 1e-11


@pytest.mark.parametrize("fn,m,N", [(homo_case, (32, 32, 32), 10), (triblock_case, (32, 32, 32), None)])
def test_pair_path_complex64(fn, m, N):
    """Compile-time passes, complex64: pair path against the two sweeps and
    the oracle over three steps."""
    from ftspolysol_b200 import Engine, FP32
    case = build(fn, m, N)
    d = derive(case)
    om, ps = case.initial_fields()
    etas = np.random.default_rng(4).standard_normal((3, len(d["modes"]) + 1, case.size)) * 0.2
    o = po.Oracle(d)
    o.set_fields(om, ps)
    ref = [o.step(e)[1] for e in etas]
    omega_ref = o.get("omega")
    o.close()
    out = []
    for on in (True, False):
        eng = Engine(d, precision=FP32)
        assert eng.set_chain_symmetry(on) == (1 if on else 0)
        eng.set_fields(om, ps)
        recs = [eng.step(e)[1] for e in etas]
        out.append((recs, eng.get("omega"), eng.get("rho_type")))
        eng.close()
        for r, rr in zip(recs, ref):
            assert rec_err(r, rr) < 2e-3
        assert rel(out[-1][1], omega_ref) < 1e-5
    (ra, wa, pa), (rb, wb, pb) = out
    assert rel(wa, wb) < 1e-5
    assert rel(pa, pb) < 1e-5
    for x, y in zip(ra, rb):
        assert rec_err(x, y) < 2e-4
