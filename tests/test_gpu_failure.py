"""Failure detection on the GPU without a fault: the bounded mbarrier wait of
the pipelined pass kernels is run on a barrier that nothing completes, with a
short limit; the wait expires, the kernel records the timeout and returns,
opfc_sync reports OPFC_ERR_TIMEOUT, and the same handle then steps on and still
matches the oracle (the context stayed usable)."""
import math
import time

import numpy as np
import pytest

import openpfc_b200 as ob
from openpfc_b200 import _lib

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3


def test_bounded_wait_expires_and_is_reported(oracle):
    n = (32, 32, 32)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 13)
    m = ob.PfcB200(n, PI4, precision=ob.FP32)
    m.initialize(0.5)
    m.set_psi(psi0)
    m.sync()
    t0 = time.perf_counter()
    assert _lib.lib().opfc_check_bounded_wait(m._h, 5.0) == 0
    with pytest.raises(ob.OpfcError) as e:
        m.sync()
    assert e.value.status == -5  # OPFC_ERR_TIMEOUT
    assert time.perf_counter() - t0 >= 0.005  # the wait ran to its limit
    m.sync()  # the status was consumed
    m.set_psi(psi0)
    m.step(5)
    m.sync()
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 5)
    assert np.linalg.norm((m.get_psi() - ref).ravel()) / np.linalg.norm(ref.ravel()) <= 1e-5


def test_bounded_wait_limit_is_checked():
    m = ob.PfcB200((16, 16, 16), PI4, precision=ob.FP32)
    assert _lib.lib().opfc_check_bounded_wait(m._h, 0.0) == -1
    assert _lib.lib().opfc_check_bounded_wait(m._h, 5000.0) == -1
