"""Learned semi-implicit preconditioner: kernels against the CPU oracle, and
what the trained network gains over the analytic (Debye) kernel.

The network, its training and its use are hand-written CUDA kernels in
libftsp (learned.cuh); oracle/mlp_oracle.py restates the same network and
loss in float64.  Tolerances: FP32 kernels against the float64 oracle, 1e-5
relative on the loss and 1e-4 of the largest gradient entry.
"""
import numpy as np
import pytest

import mlp_oracle as mo
from ftspolysol_b200 import cases
from ftspolysol_b200.derive import derive
from ftspolysol_b200.engine import Engine, FP32, FP64, SCHEME_SI, SCHEME_PC

pytestmark = pytest.mark.gpu


def pe_case(m, N=32, salt=0.1, valence=1.0, lB=1.0, dt=0.005):
    V = (m * 0.5) ** 3
    nchain = int(round(0.5 * V / N))
    return cases.Case(name="learn_%d" % m, m=(m, m, m), dL=0.5, a=1.0, monomer_names=["A"], chi=[0.0], xi=0.1,
                      lB=lB, species=[cases.homopolymer("P", nchain, N)],
                      counterions={"number": "auto_neutralize", "valence": valence},
                      salt={"num_salt": int(round(salt * V)), "cation_valence": 1.0, "anion_valence": -1.0},
                      dt=dt, init_seed=5)


def k2_grid(case):
    ks = [2 * np.pi * np.where(np.arange(n) > n // 2, np.arange(n) - n, np.arange(n)) / L for n, L in zip(case.m, case.L)]
    return (ks[0][:, None, None] ** 2 + ks[1][None, :, None] ** 2 + ks[2][None, None, :] ** 2).ravel()


def test_gradient_matches_cpu_oracle():
    case = pe_case(16, N=8)
    e = Engine(derive(case), precision=FP32, scheme=SCHEME_SI)
    e.learn_configure(N=8, lB=1.0, salt=0.1, seed=3)
    rng = np.random.default_rng(0)
    n = 300   # two full CTAs and a partial one
    x = rng.normal(size=(n, 6)).astype(np.float32)
    t = rng.normal(size=(n, 2)).astype(np.float32)
    m = (rng.random((n, 2)) > 0.3).astype(np.float32)
    w = e.learn_weights()
    assert w.size == mo.n_params(2)
    for _ in range(2):   # the same result on a second call
        loss, g = e.learn_grad(x, t, m)
        lc, gc = mo.loss_and_grad(w.astype(np.float64), x.astype(np.float64), t.astype(np.float64),
                                  m.astype(np.float64), 2)
        assert abs(loss - lc) <= 1e-5 * abs(lc)
        assert np.abs(g - gc).max() <= 1e-4 * np.abs(gc).max()
    e.close()


def test_set_dt_matches_a_handle_built_with_that_dt():
    case = pe_case(16, N=8)
    d = derive(case)
    om, ps = case.initial_fields()
    eta = np.random.default_rng(4).standard_normal((2, case.size)) * 0.1
    out = []
    for scheme in (SCHEME_PC, SCHEME_SI):
        d1 = dict(d, dt=0.01)
        d2 = dict(d, dt=0.03)
        a = Engine(d1, precision=FP64, scheme=scheme)
        b = Engine(d2, precision=FP64, scheme=scheme)
        b.set_dt(0.01)
        for e in (a, b):
            e.set_fields(om, ps)
            e.step(eta)
        np.testing.assert_array_equal(a.get("omega"), b.get("omega"))
        np.testing.assert_array_equal(a.get("psi"), b.get("psi"))
        a.close(); b.close()


@pytest.fixture(scope="module")
def trained():
    """A 32^3 polyelectrolyte solution (N = 32, monovalent counterions, salt
    0.1): 100 plain semi-implicit steps, then 400 steps collecting the
    (force, field-increment) statistics, then 1500 Adam steps."""
    case = pe_case(32)
    d = derive(case)
    om, ps = case.initial_fields()
    e = Engine(d, precision=FP32, scheme=SCHEME_SI, noise=True, seed=3, restart_interval=20)
    e.set_fields(om, ps)
    e.learn_configure(N=32, lB=1.0, salt=0.1, seed=11)
    for _ in range(100):
        e.step_async()
    e.learn_collect(True)
    for _ in range(400):
        e.step_async()
    e.learn_collect(False)
    first = e.learn_train(20)
    last = e.learn_train(1480)
    yield case, d, e, first, last
    e.close()


def test_training_reduces_the_loss(trained):
    _, _, e, first, last = trained
    assert np.isfinite(last) and last < 0.5 * first
    st = e.learn_stats()
    assert st["iterations"] == 1500
    # (wave vector, field) targets with finite, positive statistics
    assert 0.1 * 2 * 32 ** 3 < st["valid_targets"] <= 2 * 32 ** 3


def test_training_needs_valid_targets():
    """Statistics with no usable target (zero mobility and no noise: the
    predictor never moves a field, so every <|dw|^2> is zero) make
    ftsp_learn_train fail instead of returning the loss of an empty batch."""
    from ftspolysol_b200.engine import FtspError
    case = pe_case(16, N=8)
    d = derive(case)
    d = dict(d, lambda_psi=0.0, modes=[dict(m, **{"lambda": 0.0}) for m in d["modes"]])
    e = Engine(d, precision=FP32, scheme=SCHEME_SI, noise=False)
    om, ps = case.initial_fields()
    e.set_fields(om, ps)
    e.learn_configure(N=8, lB=1.0, salt=0.1, seed=3)
    e.learn_collect(True)
    for _ in range(3):
        e.step_async()
    e.learn_collect(False)
    with pytest.raises(FtspError, match="no valid training target"):
        e.learn_train(10)
    assert e.learn_stats()["valid_targets"] == 0
    e.close()


def test_network_reproduces_the_measured_response(trained):
    """What the network gains: at long wavelengths (k^2 < 4) the measured
    linear response of the drift to the field increments differs from the
    homogeneous-state Debye kernel; the trained network's coefficients track
    the measurement, the analytic ones do not.  At short wavelengths, where
    the chain response vanishes, both agree with the measurement."""
    case, _, e, _, _ = trained
    A = e.get("learn_A").real.reshape(2, -1)
    B = e.get("learn_B").real.reshape(2, -1)
    GA = e.get("si_G").real.reshape(2, -1)
    e.learn_use(True)
    GL = e.get("learned_G").real.reshape(2, -1)
    e.learn_use(False)
    k2 = k2_grid(case)
    err_l, err_a = [], []
    for f in range(2):
        ok = (A[f] > 0) & (B[f] > 0) & (GA[f] > 0) & (k2 < 4.0)
        G_meas = A[f][ok] / B[f][ok]
        err_l.append(np.abs(np.log(GL[f][ok] / G_meas)))
        err_a.append(np.abs(np.log(GA[f][ok] / G_meas)))
        hi = (A[f] > 0) & (B[f] > 0) & (GA[f] > 0) & (k2 > 9.0)
        assert np.median(np.abs(np.log(GL[f][hi] / GA[f][hi]))) < 0.05
    err_l = np.concatenate(err_l)
    err_a = np.concatenate(err_a)
    assert np.median(err_l) < 0.6 * np.median(err_a), (np.median(err_l), np.median(err_a))


def test_fallback_rule_counts(trained):
    """With a fallback ratio below any attainable residual ratio every judged
    step falls back to the analytic kernel."""
    case, d, e, _, _ = trained
    w = e.learn_weights()
    om, ps = case.initial_fields()
    f = Engine(d, precision=FP32, scheme=SCHEME_SI, noise=True, seed=5)
    f.set_fields(om, ps)
    f.learn_configure(N=32, lB=1.0, salt=0.1, seed=11, fallback_ratio=1e-12)
    f.learn_set_weights(w)
    f.learn_use(True)
    for _ in range(10):
        f.step()
    st = f.learn_stats()
    assert st["checks"] == 10 and st["fallbacks"] == 10 and st["using_learned"] == 0
    f.close()

