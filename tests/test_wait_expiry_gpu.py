"""Failure detection: a bounded device-side wait that runs out (GPU).

The one-launch triangular solve makes each 64-row block wait for the blocks
before it.  b200la_test_wait_expiry runs that solve with block 0 never
claimed, so the other blocks wait for a publication that never comes.  The
wait limit is short (a few milliseconds), the kernel records DEV_WAIT_TIMEOUT
in the workspace's status block and returns, and the host reports
B200LA_DEVICE_TIMEOUT.  Nothing faults or hangs; the next normal solve on the
same device and workspace must still be bit-identical to the oracle.
"""
import time

import numpy as np
import pytest
import torch

from linearalgebra_b200 import _lib
from linearalgebra_b200.workloads import system

pytestmark = pytest.mark.gpu


def _solve(lib, a, b, ws, nbytes, s):
    n = a.shape[0]
    m = torch.from_numpy(a).cuda()
    x = torch.from_numpy(b).cuda()
    piv = torch.empty(n, dtype=torch.int64, device="cuda")
    _lib.check(lib.b200la_dgesv(m.data_ptr(), piv.data_ptr(), n, x.data_ptr(), 1, ws.data_ptr(), nbytes, s))
    torch.cuda.synchronize()
    return m.cpu().numpy(), piv.cpu().numpy(), x.cpu().numpy()


@pytest.mark.parametrize("n", [300, 1024])
def test_expired_wait_reports_timeout_and_device_stays_usable(port, n):
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    a, _, b = system(n, seed=600 + n)
    nbytes = lib.b200la_dgesv_workspace_size(n, 1)
    ws = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    lu, piv, x_before = _solve(lib, a, b, ws, nbytes, s)

    lu_d = torch.from_numpy(lu).cuda()
    x = torch.from_numpy(b).cuda()
    t0 = time.perf_counter()
    st = lib.b200la_test_wait_expiry(lu_d.data_ptr(), n, x.data_ptr(), 5_000_000, ws.data_ptr(), nbytes, s)
    elapsed = time.perf_counter() - t0
    assert st == _lib.DEVICE_TIMEOUT, (st, _lib.last_error())
    assert "site 20" in _lib.last_error()
    assert elapsed < 1.5, f"the 5 ms waits took {elapsed:.2f} s to give up"
    assert np.array_equal(x.cpu().numpy(), b), "an aborted solve wrote x"
    # the status block keeps the error until the next operation re-initializes it
    info = torch.zeros(1, dtype=torch.int32)
    st2 = lib.b200la_workspace_status(ws.data_ptr(), info.data_ptr(), s)
    assert st2 == _lib.DEVICE_TIMEOUT

    # same device, same workspace: the next solve's factors and pivots are
    # bit-identical to the oracle, its solution to the one before the
    # expired wait, and its backward error within 10 n eps
    lu2, piv2, x2 = _solve(lib, a, b, ws, nbytes, s)
    lu_ref, piv_ref, _ = port.gesv(a, b)
    assert np.array_equal(piv2, piv_ref)
    assert np.array_equal(lu2, lu_ref)
    assert np.array_equal(x2, x_before)
    assert port.backward_error(a, x2, b) <= 10 * n * np.finfo(np.float64).eps
    assert lib.b200la_workspace_status(ws.data_ptr(), info.data_ptr(), s) == _lib.SUCCESS


def test_wait_expiry_argument_checks():
    lib = _lib.load()
    p = torch.empty(8, dtype=torch.float64, device="cuda")
    assert lib.b200la_test_wait_expiry(p.data_ptr(), 64, p.data_ptr(), 5_000_000, p.data_ptr(), 64, None) \
        == _lib.INVALID_ARGUMENT
    assert lib.b200la_test_wait_expiry(p.data_ptr(), 256, p.data_ptr(), 10, p.data_ptr(), 64, None) \
        == _lib.INVALID_ARGUMENT
