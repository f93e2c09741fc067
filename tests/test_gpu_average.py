"""Device-side time averages of the observable record.

The averaging rule is the reference's (complexLangevin.cu:424-467): steps
after the first Nss, at most Ns records, real parts.  The engine accumulates
on the device (so it runs inside the step graph and replica batches) and
adds block means for a standard error.  Checked against the same averages
taken on the host from the per-step records, 1e-12 relative, and between a
directly stepped engine and the same engine inside a replica batch (equal).
"""
import numpy as np
import pytest

from ftspolysol_b200.cases import workload
from ftspolysol_b200.derive import derive

pytestmark = pytest.mark.gpu


def make(prec, seed=9):
    from ftspolysol_b200 import Engine, FP32, FP64, SCHEME_SI
    case = workload(1)
    d = derive(case)
    om, ps = case.initial_fields()
    e = Engine(d, precision=FP64 if prec == "fp64" else FP32, scheme=SCHEME_SI, noise=True, seed=seed)
    e.set_fields(om, ps)
    return e


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_average_matches_host_records(prec):
    skip, samples, blocks = 5, 20, 4
    e = make(prec)
    e.average_start(skip, samples, blocks)
    recs = []
    for _ in range(30):
        _, rec, _ = e.step()
        recs.append(rec.real.copy())
    mean, se, n = e.average_read()
    e.close()
    assert n == samples
    used = np.array(recs[skip:skip + samples])
    np.testing.assert_allclose(mean, used.mean(axis=0), rtol=1e-12, atol=1e-14)
    bm = used.reshape(blocks, samples // blocks, -1).mean(axis=1)
    ref_se = bm.std(axis=0, ddof=1) / np.sqrt(blocks)
    np.testing.assert_allclose(se, ref_se, rtol=1e-9, atol=1e-14)


def test_average_in_a_replica_batch():
    from ftspolysol_b200.engine import Batch
    a, b = make("fp32", seed=4), make("fp32", seed=4)
    for e in (a, b):
        e.average_start(2, 12, 3)
    for _ in range(14):
        a.step_async()
    bt = Batch([b], 2)
    bt.step(7)
    bt.sync()
    bt.close()
    ma, sa, na = a.average_read()
    mb, sb, nb = b.average_read()
    a.close()
    b.close()
    assert na == nb == 12
    np.testing.assert_array_equal(ma, mb)
    np.testing.assert_array_equal(sa, sb)


def test_average_drops_records_undone_by_a_rollback():
    """A non-finite step rolls the fields back to the last checkpoint; the
    records taken since that checkpoint go with them, and only records up to
    the last checkpoint are committed to the averages."""
    from ftspolysol_b200 import Engine, FP64, SCHEME_SI
    from ftspolysol_b200.engine import NonFinite
    case = workload(1)
    d = derive(case)
    om, ps = case.initial_fields()
    every = 4
    e = Engine(d, precision=FP64, scheme=SCHEME_SI, noise=True, seed=9, restart_interval=every)
    e.set_fields(om, ps)
    e.average_start(0, 1000, 2)
    nan_eta = np.zeros((2, case.size))
    nan_eta[0, 5] = np.nan
    rows, ckpt = [], 0
    for attempt in range(1, 15):
        if attempt in (7, 10):
            e.set_noise(nan_eta)
        try:
            _, rec, _ = e.step()
        except NonFinite:
            del rows[ckpt:]
            continue
        rows.append(rec.real.copy())
        if attempt % every == 0:
            ckpt = len(rows)
    mean, _, n = e.average_read()
    e.close()
    kept = np.array(rows[:ckpt])
    assert n == len(kept)
    np.testing.assert_allclose(mean, kept.mean(axis=0), rtol=1e-12, atol=1e-14)
