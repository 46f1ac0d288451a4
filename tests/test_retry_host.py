"""The oracle's restatement of the model's retry protocol (CPU)."""
import numpy as np


def test_retry_protocol_accumulates(pkg, orc):
    b = pkg.workloads.plain_small(12, seed=31, warm_h=True)
    b.ICNTRL[3, :] = 140
    b.RTOL[:] = 2e-3
    C1, ist1, rst1, ierr1 = orc.integrate_batch(b)
    C, ist, rst, ierr, nf1, nf2 = orc.integrate_with_retry(
        b, np.full(b.ATOL.shape, 1e-2), np.full(b.RTOL.shape, 0.5e-2))
    fail = ierr1 < 0
    assert nf1 == int(fail.sum()) > 0 and nf2 == 0
    assert (ierr == 1).all()
    # counters of retried cells add both attempts; others are untouched
    assert (ist[:, fail] > ist1[:, fail]).any()
    assert np.array_equal(ist[:, ~fail], ist1[:, ~fail])
    assert np.array_equal(C[:, ~fail], C1[:, ~fail])
