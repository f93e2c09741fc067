"""The MLP oracle's back-propagation against central finite differences
(float64), and its Adam step against the update rule written out."""
import numpy as np

import mlp_oracle as mo


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    nout = 2
    w = rng.normal(size=mo.n_params(nout)) * 0.2
    x = rng.normal(size=(37, mo.NIN))
    t = rng.normal(size=(37, nout))
    m = (rng.random((37, nout)) > 0.2).astype(float)
    _, g = mo.loss_and_grad(w, x, t, m, nout)
    idx = rng.choice(len(w), 60, replace=False)
    # every parameter block is represented
    idx = np.concatenate([idx, [0, mo.H * mo.NIN, mo.H * mo.NIN + mo.H + 5, len(w) - 1, len(w) - nout - 3]])
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mo.loss_and_grad(wp, x, t, m, nout)[0] - mo.loss_and_grad(wm, x, t, m, nout)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 * max(1.0, abs(fd)), (i, fd, g[i])


def test_loss_definition_and_adam():
    rng = np.random.default_rng(1)
    nout = 3
    w = rng.normal(size=mo.n_params(nout)) * 0.1
    x = rng.normal(size=(5, mo.NIN))
    t = rng.normal(size=(5, nout))
    m = np.ones((5, nout))
    z, _, _ = mo.forward(w, x, nout)
    loss, g = mo.loss_and_grad(w, x, t, m, nout)
    assert np.isclose(loss, ((z - t) ** 2).mean())
    w1, m1, m2 = mo.adam_step(w, g, np.zeros_like(w), np.zeros_like(w), 1, 1e-3)
    # first bias-corrected Adam step moves every weight by lr * sign(g)
    moved = np.abs(w1 - w)
    np.testing.assert_allclose(moved[np.abs(g) > 1e-4], 1e-3, rtol=1e-3)
