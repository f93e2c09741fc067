"""Replica batches (one CUDA graph per batch step) against the same engines
stepped one by one: the graph replays the same kernels per replica, so the
fields must agree bit for bit, with fresh noise on every replay."""
import numpy as np
import pytest

from ftspolysol_b200 import cases
from ftspolysol_b200.derive import derive
from ftspolysol_b200.engine import Batch, Engine, FP32, FP64, SCHEME_PC, SCHEME_SI

pytestmark = pytest.mark.gpu


def small(m, N, seed):
    V = float(np.prod(m)) * 0.125
    return cases.Case(name="b%d" % seed, m=m, dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1, lB=1.0,
                      species=[cases.homopolymer("P", max(1, int(round(0.5 * V / N))), N)],
                      counterions={"number": "auto_neutralize", "valence": 1.0},
                      salt={"num_salt": int(round(0.1 * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                      dt=0.005, stress=("xx", "yz"), isotropic_pressure=True, init_seed=seed)


def make(case, prec, scheme, seed):
    e = Engine(derive(case), precision=prec, scheme=scheme, noise=True, seed=seed, restart_interval=4)
    om, ps = case.initial_fields()
    e.set_fields(om, ps)
    return e


@pytest.mark.parametrize("prec,scheme,spg", [(FP64, SCHEME_PC, 1), (FP32, SCHEME_SI, 2)])
def test_batch_matches_individual_steps(prec, scheme, spg):
    cs = [small((16, 16, 16), 8, 1), small((12, 8, 16), 6, 2), small((32, 32, 32), 10, 3)]
    steps = 8
    ind = [make(c, prec, scheme, 100 + k) for k, c in enumerate(cs)]
    for _ in range(steps):
        for e in ind:
            e.step_async()
    grp = [make(c, prec, scheme, 100 + k) for k, c in enumerate(cs)]
    b = Batch(grp, spg)
    assert b.launches_per_graph > 100 * len(cs) * spg
    for _ in range(2):   # two calls in a row
        b.step(steps // spg // 2)
    b.sync()
    b.close()
    for a, g in zip(ind, grp):
        for name in ("omega", "psi", "rho_type"):
            np.testing.assert_array_equal(a.get(name), g.get(name))
        sa, ra, _ = a.read_status()
        sg, rg, _ = g.read_status()
        assert sa == sg
        np.testing.assert_array_equal(ra, rg)
    # after the batch is gone the engines step on their own again
    for e in grp:
        e.step()
    for e in ind + grp:
        e.close()


def test_replays_draw_fresh_noise():
    c = small((16, 16, 16), 8, 4)
    e = make(c, FP64, SCHEME_PC, 9)
    b = Batch([e], 1)
    b.step(1)
    b.sync()
    w1 = e.get("omega").copy()
    b.step(1)
    b.sync()
    w2 = e.get("omega")
    b.close()
    # the second replay moved the field by a different noise realisation
    ref = make(c, FP64, SCHEME_PC, 9)
    ref.step_async()
    np.testing.assert_array_equal(ref.get("omega"), w1)
    ref.step_async()
    np.testing.assert_array_equal(ref.get("omega"), w2)
    assert not np.array_equal(w1, w2)
    e.close()
    ref.close()
