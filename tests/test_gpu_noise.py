"""Moments of the engine's Langevin noise (the Philox path every long run uses).

The reference draws, every step, real Gaussian noise of variance
sigma^2 = 2 lambda dt / dV for each interaction mode and for psi
(generate_noises, complexLangevin.cu:287-297; langevin_noise_stddev,
common.h:300-303, generateNoiseKernel, common.h:582-590) and removes the mean
of the psi noise (remove_real_mean, complexLangevin.cu:296).  The engine
draws the same distribution from a counter-based Philox4x32-10 generator
keyed by (seed, step, field pair, point), whose two Box-Muller outputs are
the noise of the two fields of the pair.  Checked here over several steps
of a 32^3 system, for both precisions:

  * mean and variance of every field against 0 and sigma^2, within 5
    standard errors (the variance of a sample variance is 2 sigma^4 / n);
  * the excess kurtosis against 0 (a Gaussian; standard error sqrt(24/n));
  * the psi noise has zero mean after the removal (to rounding);
  * no correlation between consecutive steps, nor between the mode and psi
    noise of one step, nor between their squares (the two outputs of one
    Box-Muller draw are independent, not only uncorrelated) (|r| < 5 / sqrt(n));
  * the same seed reproduces the noise exactly, another seed does not.
"""
import numpy as np
import pytest

from ftspolysol_b200.cases import workload
from ftspolysol_b200.derive import derive

pytestmark = pytest.mark.gpu

STEPS = 6


def draws(prec, seed, dt=0.005):
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_PC
    case = workload(1)
    d = dict(derive(case), dt=dt)
    om, ps = case.initial_fields()
    e = Engine(d, precision=FP64 if prec == "fp64" else FP32, scheme=SCHEME_PC, noise=True, seed=seed)
    e.set_fields(om, ps)
    out = []
    for _ in range(STEPS):
        e.step()
        out.append(e.get("eta").real.reshape(2, -1).copy())
    e.close()
    return d, np.array(out)   # (steps, fields, points)


def corr(a, b):
    a = a - a.mean()
    b = b - b.mean()
    return float(np.dot(a, b) / np.sqrt(np.dot(a, a) * np.dot(b, b)))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_noise_moments(prec):
    d, eta = draws(prec, seed=1234)
    n = eta.shape[2]
    lam = [d["modes"][0]["lambda"], d["lambda_psi"]]
    for f in range(2):
        sigma2 = 2.0 * lam[f] * d["dt"] / d["dV"]
        x = eta[:, f, :].reshape(-1)
        N = x.size
        if f == 0:
            assert abs(x.mean()) < 5.0 * np.sqrt(sigma2 / N)
        var = float(np.mean(x * x))
        assert abs(var / sigma2 - 1.0) < 5.0 * np.sqrt(2.0 / N), (f, var, sigma2)
        kurt = float(np.mean(x ** 4) / var ** 2 - 3.0)
        assert abs(kurt) < 5.0 * np.sqrt(24.0 / N), (f, kurt)
    # psi noise: mean removed in every step
    tol = 1e-12 if prec == "fp64" else 1e-6
    for s in range(STEPS):
        sig = np.sqrt(2.0 * lam[1] * d["dt"] / d["dV"])
        assert abs(eta[s, 1].mean()) < tol * sig
    # independence across steps and between fields
    bound = 5.0 / np.sqrt(n)
    for f in range(2):
        for s in range(STEPS - 1):
            assert abs(corr(eta[s, f], eta[s + 1, f])) < bound
    for s in range(STEPS):
        assert abs(corr(eta[s, 0], eta[s, 1])) < bound
        assert abs(corr(eta[s, 0] ** 2, eta[s, 1] ** 2)) < bound


def test_noise_seeded():
    _, a = draws("fp64", seed=77)
    _, b = draws("fp64", seed=77)
    _, c = draws("fp64", seed=78)
    np.testing.assert_array_equal(a, b)
    assert abs(corr(a[0, 0], c[0, 0])) < 5.0 / np.sqrt(a.shape[2])


def test_noise_follows_dt():
    """sigma^2 is proportional to dt (common.h:300-303)."""
    d1, a = draws("fp64", seed=5, dt=0.005)
    d2, b = draws("fp64", seed=5, dt=0.02)
    r = float(np.mean(b[:, 0] ** 2) / np.mean(a[:, 0] ** 2))
    assert abs(r / 4.0 - 1.0) < 0.02
