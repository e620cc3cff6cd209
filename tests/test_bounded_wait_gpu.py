"""A bounded wait on global memory that runs out: the radius search computes
its output offsets with a chained scan in which every group of 32 pieces
waits for the groups before it.  AOCLDA_B200_TEST_RADIUS_WAIT=1 keeps the
first group from publishing its count -- a flag that nothing sets -- and
shortens the waits; every waiting group gives up at its limit and the call returns
da_status_internal_error instead of hanging.  The same handle, and a fresh
one, then search normally: the device stays usable."""
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

INTERNAL_ERROR = 1
ENV = "AOCLDA_B200_TEST_RADIUS_WAIT"


def test_radius_offset_scan_wait_runs_out(gpu, ab):
    rng = np.random.default_rng(8)
    X = rng.standard_normal((40_000, 8))  # three 16,384-column chunks per query row
    Q = rng.standard_normal((30, 8))
    nn = ab.KNN("d", order=ab.ROW_MAJOR).fit(X)
    want = nn.radius_neighbors(Q, 1.5, True, True)
    os.environ[ENV] = "1"
    try:
        t = time.perf_counter()
        with pytest.raises(ab.DAError) as ei:
            nn.radius_neighbors(Q, 1.5, True, True)
        assert time.perf_counter() - t < 30.0
        assert ei.value.status == INTERNAL_ERROR
    finally:
        os.environ.pop(ENV, None)
    again = nn.radius_neighbors(Q, 1.5, True, True)
    nn.close()
    fresh = ab.KNN("d", order=ab.ROW_MAJOR).fit(X)
    third = fresh.radius_neighbors(Q, 1.5, True, True)
    fresh.close()
    for got in (again, third):
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)
