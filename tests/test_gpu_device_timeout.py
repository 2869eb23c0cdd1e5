"""GPU: the bounded device waits give up, report MOEA_ERR_DEVICE_TIMEOUT and
leave the device usable.

Every spin of the library's kernels has a limit: the peel's front barriers
(2 s, both the counted barrier of the lane-owned peel and the grid barrier of
the general peel) and the tensor-core association's mbarrier waits (1 s).
moea_selftest_wait_timeout runs the same device routines against a condition
that never completes (a barrier that asks for one arrival more than the grid
has, an mbarrier whose one arrival never comes) with a short limit.  The test
checks the status the host reads, that the wait ended near its limit, and
that a non-dominated sort on the same workspace afterwards still matches the
oracle.  Nothing here faults or traps the GPU.
"""
import ctypes
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT_NS = 5_000_000  # 5 ms


@pytest.fixture(scope="module")
def ws():
    from cuda_moea import stages
    w = stages.Workspace(max_points=8192, max_objectives=3, max_directions=128)
    yield w
    w.close()


def _selftest(ws, which, limit_ns):
    from cuda_moea._lib import lib
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib().moea_selftest_wait_timeout(ws.handle, which, ctypes.c_ulonglong(limit_ns), stream)


@pytest.mark.parametrize("which,what", [(0, b"front peeling"), (1, b"front peeling"), (2, b"association")])
def test_wait_runs_out_and_reports_timeout(ws, oracle, which, what):
    from cuda_moea import stages
    from cuda_moea._lib import lib
    t0 = time.perf_counter()
    status = _selftest(ws, which, LIMIT_NS)
    elapsed = time.perf_counter() - t0
    assert status == 5, f"expected MOEA_ERR_DEVICE_TIMEOUT, got {status}"
    assert what in lib().moea_last_error()
    assert elapsed < 1.0, f"the wait took {elapsed:.3f} s against a {LIMIT_NS / 1e6:.0f} ms limit"

    # the status word was cleared and the workspace sorts correctly afterwards
    rng = np.random.default_rng(which)
    objs = rng.random((3, 4000)).astype(np.float32)
    cv = np.zeros(4000, np.float32)
    got, mf = stages.ndsort(ws, torch.from_numpy(cv).cuda(), torch.from_numpy(objs).cuda(), 2000)
    want, wmf = oracle.ndsort(cv, objs, 2000)
    assert mf == wmf
    assert np.array_equal(got.cpu().numpy(), want)


def test_limit_is_validated(ws):
    assert _selftest(ws, 0, 0) == 1
    assert _selftest(ws, 3, LIMIT_NS) == 1
    assert _selftest(ws, 2, 3_000_000_000) == 1
