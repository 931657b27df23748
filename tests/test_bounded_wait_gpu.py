"""The bounded waits of the decoupled look-back (csrc/scan.cuh), made to run out on purpose.

A scan tile waits for its predecessors to publish; every wait gives up after a fixed number of
polls, records GTSC_ERR_TIMEOUT in the scan's error word and returns, so that a predecessor that
never publishes cannot hang the GPU.  gtsc_selftest_lookback_timeout runs one look-back whose
predecessor is never published (a flag that nothing sets): the wait must end by itself with
GTSC_ERR_TIMEOUT, and the device must stay usable for the next call.
"""
import numpy as np
import pytest

import oracle as OR

pytestmark = pytest.mark.gpu

ERR_TIMEOUT = -7


def test_lookback_wait_runs_out_and_the_device_stays_usable(G):
    err, seconds = G.selftest_lookback_timeout()
    assert err == ERR_TIMEOUT, G.STATUS_NAMES.get(err, err)
    assert 0.0 < seconds < 60.0, seconds
    # the context is still usable: an ordinary encode and decode right after
    x = np.arange(1 << 16, dtype=np.int32) * 3
    parts = G.encode(OR.DELTA, OR.INT, G.to_device(x))
    back = G.to_host(G.decode(OR.DELTA, OR.INT, parts), np.int32)
    assert np.array_equal(back, x)
