"""ftsp_step through the captured step graph against the same steps launched
kernel by kernel: bit-identical fields, records and status, including a
change of dt, the adaptive step, injected noise (which launches directly),
the two schemes and both precisions."""
import numpy as np
import pytest

from ftspolysol_b200 import cases
from ftspolysol_b200.derive import derive
from ftspolysol_b200.engine import Engine, FP32, FP64, SCHEME_PC, SCHEME_SI

pytestmark = pytest.mark.gpu


def case(m, N):
    V = float(np.prod(m)) * 0.125
    return cases.Case(name="g", m=m, dL=0.5, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
                      species=[cases.homopolymer("P", max(1, int(round(0.5 * V / N))), N)],
                      counterions={"number": "auto_neutralize", "valence": 1.0},
                      salt={"num_salt": int(round(0.1 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                      dt=0.005, stress=("xx", "xy"), isotropic_pressure=True, init_seed=2)


@pytest.mark.parametrize("prec,scheme,m", [(FP64, SCHEME_PC, (16, 12, 10)), (FP32, SCHEME_SI, (32, 32, 32))])
def test_step_graph_is_bit_identical(prec, scheme, m):
    c = case(m, 8)
    d = derive(c)
    om, ps = c.initial_fields()
    engs = []
    for graph in (True, False):
        e = Engine(d, precision=prec, scheme=scheme, noise=True, seed=21, restart_interval=3)
        e.set_step_graph(graph)
        e.set_fields(om, ps)
        engs.append(e)
    eta = np.random.default_rng(5).standard_normal((2, c.size)) * 0.1

    def both(fn):
        return [fn(e) for e in engs]

    for k in range(14):
        if k == 5:
            both(lambda e: e.set_dt(0.004))
        if k == 8:
            both(lambda e: e.set_adaptive(0.5))
        if k == 11:
            outs = both(lambda e: e.step(eta))      # injected noise
        else:
            outs = both(lambda e: e.step())
        (qa, ra, da), (qb, rb, db) = outs
        np.testing.assert_array_equal(qa, qb)
        np.testing.assert_array_equal(ra, rb)
        np.testing.assert_array_equal(da, db)
    for name in ("omega", "psi", "rho_type"):
        np.testing.assert_array_equal(engs[0].get(name), engs[1].get(name))
    assert engs[0].launches() == engs[1].launches()
    assert engs[0].restarts() == engs[1].restarts()
    for e in engs:
        e.close()
