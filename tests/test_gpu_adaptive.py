"""Adaptive step (dt_eff = dt min(1, u_ref / max|u|)): identical to the fixed
step when the bound is never reached, equal to a fixed step of dt_eff when it
is, and the noise amplitude follows dt_eff."""
import numpy as np
import pytest

from ftspolysol_b200 import cases
from ftspolysol_b200.derive import derive
from ftspolysol_b200.engine import Engine, FP64, SCHEME_PC, SCHEME_SI

pytestmark = pytest.mark.gpu


def small(seed=3):
    V = 16.0 ** 3 * 0.125
    return cases.Case(name="ad", m=(16, 16, 16), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
                      species=[cases.homopolymer("P", int(round(0.5 * V / 8)), 8)],
                      counterions={"number": "auto_neutralize", "valence": 1.0},
                      salt={"num_salt": int(round(0.1 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                      dt=0.01, stress=("xx",), isotropic_pressure=True, init_seed=seed)


@pytest.mark.parametrize("scheme", [SCHEME_PC, SCHEME_SI])
def test_unreached_bound_changes_nothing(scheme):
    c = small()
    d = derive(c)
    om, ps = c.initial_fields()
    a = Engine(d, precision=FP64, scheme=scheme, noise=True, seed=5)
    b = Engine(d, precision=FP64, scheme=scheme, noise=True, seed=5)
    b.set_adaptive(1e30)
    for e in (a, b):
        e.set_fields(om, ps)
        for _ in range(3):
            e.step()
    np.testing.assert_array_equal(a.get("omega"), b.get("omega"))
    np.testing.assert_array_equal(a.get("psi"), b.get("psi"))
    dt_eff, umax = b.step_info()
    assert dt_eff == 0.01 and umax > 0
    a.close(); b.close()


@pytest.mark.parametrize("scheme", [SCHEME_PC, SCHEME_SI])
def test_reached_bound_is_a_step_of_dt_eff(scheme):
    c = small()
    d = derive(c)
    om, ps = c.initial_fields()
    probe = Engine(d, precision=FP64, scheme=scheme, noise=True, seed=9)
    probe.set_fields(om, ps)
    probe.set_adaptive(1e30)
    probe.step()
    _, umax = probe.step_info()
    probe.close()
    a = Engine(d, precision=FP64, scheme=scheme, noise=True, seed=9)
    a.set_adaptive(0.25 * umax)
    a.set_fields(om, ps)
    a.step()
    dt_eff, um = a.step_info()
    assert um == pytest.approx(umax, rel=1e-14)
    assert dt_eff == pytest.approx(0.0025, rel=1e-12)
    b = Engine(dict(d, dt=dt_eff), precision=FP64, scheme=scheme, noise=True, seed=9)
    b.set_fields(om, ps)
    b.step()
    for name in ("omega", "psi"):
        x, y = a.get(name), b.get(name)
        assert np.max(np.abs(x - y)) <= 1e-12 * np.max(np.abs(y))
    a.close(); b.close()
