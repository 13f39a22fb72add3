"""The allocation-free forward transform (opfc_fft_forward_noalloc) against the
handle-based opfc_fft_forward and the FP64 oracle, through the C ABI.

It exists for callers that cannot allocate device memory: latency-bound loops
that cannot absorb cudaMalloc's device-wide synchronisation, and host
applications whose own allocator owns every device allocation.  Its scratch is
a fixed 16 MiB array inside the library, shared by all calls.  Two calls in a
row must both match the handle path and the oracle; sizes beyond the array are
refused.  This file is collected last so a failure here never hides the other
tests, and it passes alone in a fresh process as well as after them.
"""
import ctypes

import numpy as np
import pytest

import openpfc_b200 as ob
from openpfc_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = {ob.FP64: 1e-12, ob.FP32: 2e-6}


def _noalloc(x_dev, out_dev, n, prec):
    import torch
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nn = (ctypes.c_int * 3)(*n)
    return _lib.lib().opfc_fft_forward_noalloc(ctypes.c_void_p(x_dev.data_ptr()),
                                               ctypes.c_void_p(out_dev.data_ptr()), nn, prec, stream)


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
@pytest.mark.parametrize("n", [(64, 48, 32), (128, 64, 64), (32, 32, 32)])
def test_noalloc_matches_handle_path_twice(oracle, prec, n):
    import torch
    tdt = torch.float64 if prec == ob.FP64 else torch.float32
    f = ob.B200Fft(n, precision=prec)
    for call in range(2):
        x = np.random.default_rng(100 + call).standard_normal((n[2], n[1], n[0]))
        x_dev = torch.tensor(x, dtype=tdt, device="cuda")
        out_dev = torch.full((n[2], n[1], n[0] // 2 + 1, 2), float("nan"), dtype=tdt, device="cuda")
        assert _noalloc(x_dev, out_dev, n, prec) == 0
        torch.cuda.synchronize()
        got = out_dev.cpu().numpy()
        got = got[..., 0] + 1j * got[..., 1]
        ref_dev = torch.zeros_like(out_dev)
        f.forward(x_dev, ref_dev)
        ref = ref_dev.cpu().numpy()
        ref = ref[..., 0] + 1j * ref[..., 1]
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= TOL[prec], (call, err)
        # and the FP64 oracle's transform of the same input (values as the
        # device holds them)
        xo = x_dev.cpu().numpy().astype(np.float64)
        ora = oracle.r2c(xo)
        err_o = np.abs(got - ora).max() / np.abs(ora).max()
        assert err_o <= TOL[prec], (call, err_o)


def test_noalloc_rejects_sizes_beyond_its_array():
    import torch
    x = torch.zeros(8, device="cuda")
    # (129 * 256 * 256) complex FP32 = 67.6 MB > 16 MiB
    assert _noalloc(x, x, (256, 256, 256), ob.FP32) == -2
    # 2048 > longest supported axis of the twiddle area
    assert _noalloc(x, x, (2048, 2, 2), ob.FP32) == -2
    assert _noalloc(x, x, (7, 8, 8), ob.FP32) == -2
