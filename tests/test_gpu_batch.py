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
    assert b.launches_per_graph > 40 * len(cs) * spg   # a whole step per replica (forward sweep alone: ~90 launches)
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


def test_autotuner_picks_a_geometry_and_keeps_results():
    """48^3 runs the runtime-plan passes: the tuner times the alternatives,
    keeps the fastest, caches it for the next handle of the same grid, and
    the step agrees with the default geometry to round-off (complex128)."""
    c = small((48, 48, 48), 8, 5)
    d = derive(c)
    om, ps = c.initial_fields()
    eta = np.random.default_rng(2).standard_normal((2, c.size)) * 0.1
    runs = []
    for tune in (False, True, True):
        e = Engine(d, precision=FP64, scheme=SCHEME_PC, autotune=tune)
        e.set_fields(om, ps)
        e.step(eta)
        runs.append((e.tune_info(), e.get("omega"), e.get("rho_type")))
        e.close()
    t0, t1, t2 = (r[0] for r in runs)
    assert t0["tuned"] == 0 and t1["tuned"] == 1 and t1["candidates"] >= 3
    assert t1["best_ms"] <= t1["default_ms"]
    assert t2["cached"] == 1 and (t2["max_radix"], t2["tile_width"]) == (t1["max_radix"], t1["tile_width"])
    for r in runs[1:]:
        for a, b in zip(r[1:], runs[0][1:]):
            assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(b))
    e = Engine(derive(small((32, 32, 32), 8, 6)), precision=FP32, scheme=SCHEME_SI, autotune=True)
    assert e.tune_info()["compile_time"] == 1
    e.close()
