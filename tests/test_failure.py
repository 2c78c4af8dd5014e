"""Failure detection on the GPU without a fault: the bounded device wait of
the generation kernels is made to run out (rf_context_selftest_timeout: a
wait on an mbarrier phase nothing completes, 50 ms limit); the kernel raises
the context's error word and returns, the host reports RF_ETIMEDOUT, and the
context generates correctly afterwards."""
import time

import numpy as np
import pytest

import randomfield_b200 as rf
from tests.helpers import errors, grid

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_context_recovers():
    ctx = rf.Context(0)
    torch = pytest.importorskip("torch")
    t0 = time.perf_counter()
    with pytest.raises(rf.RandomFieldError) as e:
        ctx.selftest_timeout(50.0)
    dt = time.perf_counter() - t0
    assert e.value.code == -22 and "wait expired" in str(e.value)
    assert 0.05 <= dt < 5.0
    # the same context still generates, and its error word was cleared
    x = grid(12, 0.1)
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    a = torch.empty((4, x.shape[0]), dtype=torch.float64, device="cuda")
    ctx.generate(dx, 3, x.shape[0], 1, 1, (1.0, 1.0, 1.0), 0.0, 1.0, 4, 2, a, precision="bf16", k_nstep=(8, 8, 8))
    ctx.synchronize()
    ref = rf.create_standard_gaussian_field_unstruct(x.T, 1, 1, (1.0, 1.0, 1.0), 0.0, 1.0, 4, 2, precision="bf16",
                                                     k_nstep=(8, 8, 8))
    assert errors(a.cpu().numpy().T, np.asarray(ref))[1] <= 1e-12
    ctx.close()
