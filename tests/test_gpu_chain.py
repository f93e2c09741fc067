"""ftsp_propagate_chain against a plain FP64 restatement (numpy FFTs).

q_1 = exp(-w), q_{s+1} = exp(-w) * IFFT[Phi * FFT[q_s] / V], Q = mean(q_N)
(polymer.cu:396-426).  Tolerance 1e-12 relative to the field's max modulus.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def reference_chain(w, L, N, b):
    m = w.shape
    k = [2 * np.pi * np.fft.fftfreq(mi, d=Li / mi) for mi, Li in zip(m, L)]
    k2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    phi = np.exp(-b * b * k2 / 6.0)
    e = np.exp(-w)
    q = e.copy()
    for _ in range(N - 1):
        q = e * np.fft.ifftn(phi * np.fft.fftn(q))
    return q, q.mean()


@pytest.mark.parametrize("m,N,b", [((32, 32, 32), 7, 1.0), ((12, 8, 16), 5, 1.3), ((64, 64, 64), 3, 0.8),
                                   ((16, 16, 16), 1, 1.0)])
def test_propagate_chain(m, N, b):
    import torch
    from ftspolysol_b200 import Engine
    from ftspolysol_b200.cases import Case, homopolymer
    from ftspolysol_b200.derive import derive
    case = Case(name="chain", m=m, dL=0.5, species=[homopolymer("P", 4, 4, charge=0.0)], lB=0.0,
                ions_enabled=False)
    eng = Engine(derive(case))
    rng = np.random.default_rng(5)
    w = (0.3 * rng.standard_normal(m) + 0.2j * rng.standard_normal(m)).astype(np.complex128)
    wd = torch.from_numpy(w.reshape(-1)).cuda()
    qd = torch.zeros_like(wd)
    Q = eng.propagate_chain(wd.data_ptr(), N, b, qd.data_ptr())
    torch.cuda.synchronize()
    q_ref, Q_ref = reference_chain(w, case.L, N, b)
    q = qd.cpu().numpy().reshape(m)
    assert np.max(np.abs(q - q_ref)) / np.max(np.abs(q_ref)) < 1e-12
    assert abs(Q - Q_ref) / abs(Q_ref) < 1e-12
    # the second call reuses the cached bond table and must agree exactly
    Q2 = eng.propagate_chain(wd.data_ptr(), N, b, qd.data_ptr())
    assert Q2 == Q
    eng.close()
