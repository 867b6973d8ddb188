"""Failure detection without a GPU fault: every device wait of the library
is bounded.  w2d_wait_selftest launches a kernel whose barrier nothing
completes; the wait runs out, the kernel reports W2D_ERR_TIMEOUT through
the context's error word and ends, the host reads the status, and the
context goes on working: the run continues bit for bit as if nothing had
happened.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W2D_ERR_TIMEOUT = 6


@pytest.mark.parametrize("graphs", [False, True])
def test_bounded_wait_reports_timeout_and_the_context_stays_usable(graphs):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    a, b = Simulation(p, ic), Simulation(p, ic)
    for s in (a, b):
        s.ctx.set_graphs(graphs)
        s.run(5)
    t0 = time.perf_counter()
    rc, msg = a.ctx.wait_selftest()
    took = time.perf_counter() - t0
    print(f"bounded wait gave up after {took:.2f} s: {msg!r}")
    assert rc == W2D_ERR_TIMEOUT, (rc, msg)
    assert "wait" in msg
    assert took < 10.0
    # the error word was cleared: the run goes on and equals the one that
    # never met the timeout
    for s in (a, b):
        s.run(5)
    assert a.status()["dt"] == b.status()["dt"]
    ia, ua = a.blocks()
    ib, ub = b.blocks()
    assert np.array_equal(ia, ib)
    m = np.ones((20, 20), bool)
    for r in (0, 1, 18, 19):
        for c in (0, 1, 18, 19):
            m[r, c] = False
    assert np.array_equal(ua[:, :, m], ub[:, :, m])
    # a second self-test reports again
    assert a.ctx.wait_selftest()[0] == W2D_ERR_TIMEOUT
