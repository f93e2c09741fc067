"""Field uploads that overlap the running step (ftsp_set_fields_async).

The upload goes to a device staging buffer on a copy stream and is installed
by the next call that uses the fields, with the same effect as
ftsp_set_fields: the steps that follow must be bit-identical, whether the
upload overlaps a step in flight or not, and a synchronous set_fields
supersedes an upload not yet installed.
"""
import numpy as np
import pytest

from ftspolysol_b200.cases import workload
from ftspolysol_b200.derive import derive

pytestmark = pytest.mark.gpu


def pinned(om, ps):
    import torch
    n = om.size + ps.size
    host = torch.empty(2 * n, dtype=torch.float64, pin_memory=True)
    host.numpy()[:] = np.concatenate([np.asarray(om).reshape(-1), np.asarray(ps).reshape(-1)]).view(np.float64)
    return host, host.data_ptr(), host.data_ptr() + om.size * 16


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_async_upload_matches_set_fields(prec):
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    case = workload(1)
    d = derive(case)
    om, ps = case.initial_fields()
    om2 = om * 0.5 + 0.01
    p = FP64 if prec == "fp64" else FP32
    ref = Engine(d, precision=p, scheme=SCHEME_SI, noise=True, seed=3, restart_interval=5)
    eng = Engine(d, precision=p, scheme=SCHEME_SI, noise=True, seed=3, restart_interval=5)
    h1, o1, p1 = pinned(om, ps)
    h2, o2, p2 = pinned(om2, ps)
    # reference: synchronous uploads
    ref.set_fields(om, ps)
    out_ref = [ref.step()[1]]
    ref.set_fields(om2, ps)
    out_ref.append(ref.step()[1])
    out_ref.append(ref.step()[1])
    # the same through async uploads, the second one overlapping a step in flight
    eng.set_fields_async_ptr(o1, p1)
    eng.step_async()
    eng.set_fields_async_ptr(o2, p2)        # copy runs beside the step
    st, r0, _ = eng.read_status()
    eng.step_async()                        # installs om2, then steps
    st1, r1, _ = eng.read_status()
    _, r2, _ = eng.step()
    for a, b in zip(out_ref, [r0, r1, r2]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(ref.get("omega"), eng.get("omega"))
    # a synchronous upload supersedes a pending one
    eng.set_fields_async_ptr(o2, p2)
    eng.set_fields(om, ps)
    ref.set_fields(om, ps)
    np.testing.assert_array_equal(ref.step()[1], eng.step()[1])
    ref.close()
    eng.close()
