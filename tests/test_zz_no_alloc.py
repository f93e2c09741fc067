"""The allocation-free chain propagation against the allocating one.

ftsp_propagate_chain_noalloc serves callers that cannot call cudaMalloc:
code inside a framework whose caching allocator owns the device memory, and
loops that must not wait on the allocator.  Its scratch is one static device
array inside the library, so this test checks that two calls in a row (which
reuse that array) each reproduce ftsp_propagate_chain, the handle-based entry
point that allocates its scratch, to the FP64 tolerance of the other chain
tests (1e-12 relative), that the second call leaves the device's free memory
unchanged (the driver's own count, so any allocation would show), and that
meshes beyond the stated limit are refused.
This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("m,N,b", [((32, 32, 32), 6, 1.0), ((12, 8, 16), 4, 1.2), ((64, 64, 64), 3, 0.9)])
def test_noalloc_matches_allocating_entry_point(m, N, b):
    import torch
    from ftspolysol_b200 import Engine
    from ftspolysol_b200.cases import Case, homopolymer
    from ftspolysol_b200.derive import derive
    from ftspolysol_b200.engine import last_error, propagate_chain_noalloc

    case = Case(name="noalloc", m=m, dL=0.5, species=[homopolymer("P", 4, 4, charge=0.0)], lB=0.0,
                ions_enabled=False)
    rng = np.random.default_rng(9)
    w = (0.3 * rng.standard_normal(m) + 0.2j * rng.standard_normal(m)).astype(np.complex128).reshape(-1)
    wd = torch.from_numpy(w).cuda()
    q_ref = torch.zeros_like(wd)
    eng = Engine(derive(case))
    Q_ref = eng.propagate_chain(wd.data_ptr(), N, b, q_ref.data_ptr())
    eng.close()
    for call in range(2):
        q = torch.full_like(wd, complex("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc, Q = propagate_chain_noalloc(m, case.L, wd.data_ptr(), N, b, q.data_ptr())
        assert rc == 0, last_error()
        torch.cuda.synchronize()
        if call == 1:   # the first call may load the library's kernels; a repeat call takes nothing
            assert torch.cuda.mem_get_info()[0] == free0
        err_q = float((q - q_ref).abs().max() / q_ref.abs().max())
        assert err_q < TOL, (call, err_q)
        assert abs(Q - Q_ref) / abs(Q_ref) < TOL, (call, Q, Q_ref)


def test_noalloc_rejects_meshes_beyond_the_limit():
    import torch
    from ftspolysol_b200.engine import last_error, propagate_chain_noalloc
    dummy = torch.zeros(4, dtype=torch.complex128, device="cuda")
    rc, _ = propagate_chain_noalloc((128, 128, 128), (64.0, 64.0, 64.0), dummy.data_ptr(), 3, 1.0, dummy.data_ptr())
    assert rc == 2
    assert "limit" in last_error()
    rc, _ = propagate_chain_noalloc((512, 8, 8), (256.0, 4.0, 4.0), dummy.data_ptr(), 3, 1.0, dummy.data_ptr())
    assert rc == 2
    assert "limit" in last_error()
