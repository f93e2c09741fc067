"""Compile-time (production-size) kernels against the oracle.

Grids whose extents are 32, 64 or 128 run the specialised passes (plane,
strided, z-line); other 2/3/5-smooth grids run the runtime-plan passes.
FP64 tolerance 1e-10 (fields, relative to the field's max modulus; records
relative with a 1e-3 floor); complex64 tolerance 1e-5 on fields and 2e-3 on
records (FP64 reductions over complex64 fields).
"""
import numpy as np
import pytest

import pyoracle as po
from ftspolysol_b200.cases import Case, homopolymer
from ftspolysol_b200.derive import derive

pytestmark = pytest.mark.gpu


def pe_case(m, N, seed=3):
    V = (m[0] * 0.5) * (m[1] * 0.5) * (m[2] * 0.5)
    return Case(name="pe_%dx%dx%d" % tuple(m), m=m, dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1,
                lB=1.0, species=[homopolymer("P", 2 * max(1, int(round(0.25 * V / N))), N)],
                counterions={"number": "auto_neutralize", "valence": 2.0},
                salt={"num_salt": int(round(0.05 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                dt=0.01, stress=("xx", "yy", "zz", "xy", "xz", "yz"), isotropic_pressure=True, init_seed=seed)


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(float(np.max(np.abs(b))), 1e-300))


def rec_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3)))


GRIDS = [((32, 32, 32), 8), ((64, 64, 64), 6), ((128, 32, 32), 6), ((32, 64, 64), 5), ((128, 128, 128), 3),
         # runtime-plan passes with radix-16 lengths along x and y (16, 128, 256)
         # and mixed 2/3/5 factors
         ((16, 12, 8), 4), ((128, 24, 20), 3), ((48, 16, 30), 3), ((256, 10, 9), 2)]


@pytest.mark.parametrize("m,N", GRIDS)
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_step_matches_oracle(m, N, prec):
    from ftspolysol_b200 import Engine, FP32, FP64
    case = pe_case(m, N)
    d = derive(case)
    om, ps = case.initial_fields()
    eta = np.random.default_rng(11).standard_normal((2, case.size)) * 0.2
    o = po.Oracle(d)
    o.set_fields(om, ps)
    Q0 = o.compute_densities(0)
    rho0 = o.get("rho_type")
    rec0 = o.measure(0, Q0)
    o.set_fields(om, ps)
    Qb, recb, dmb = o.step(eta)
    omega1 = o.get("omega")
    psi1 = o.get("psi")
    o.close()
    ftol, rtol = (1e-10, 1e-10) if prec == "fp64" else (1e-5, 2e-3)
    eng = Engine(d, precision=FP64 if prec == "fp64" else FP32)
    eng.set_fields(om, ps)
    assert rel(eng.compute_densities(0), Q0) < ftol
    assert rel(eng.get("rho_type"), rho0) < ftol
    assert rec_err(eng.measure(0), rec0) < rtol
    eng.set_fields(om, ps)
    Q, rec, dm = eng.step(eta)
    assert rel(Q, Qb) < ftol
    assert rec_err(rec, recb) < rtol
    assert rel(eng.get("omega"), omega1) < ftol
    assert rel(eng.get("psi"), psi1) < ftol
    eng.close()
