"""GPU parity of the stand-alone transforms (the IFFT contract) against the
FP64 oracle, through the C ABI.  Known answers from tests/unit/kernel/fft/
test_fft.cpp:28-70 and tests/unit/runtime/gpu/test_fft_cuda.cpp:84-189."""
import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

# FP64 agrees with the oracle to rounding; FP32 to its own rounding level
TOL = {ob.FP64: 1e-12, ob.FP32: 2e-6}


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_forward_dc_kat(prec):
    f = ob.B200Fft((8, 1, 1), precision=prec)
    x = np.array([0.000, 0.785, 1.571, 2.356, 3.142, 3.927, 4.712, 5.498]).reshape(1, 1, 8)
    out = f.forward(x)
    assert abs(out[0, 0, 0].real - 21.991) <= 0.01


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_backward_normalisation_kat(prec):
    f = ob.B200Fft((2, 1, 1), precision=prec)
    out = f.backward(np.array([1 + 0j, 2 + 0j]).reshape(1, 1, 2))
    assert abs(out[0, 0, 0] - 1.5) <= 0.01


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_dc_only_backward_kat(prec):
    f = ob.B200Fft((64, 64, 64), precision=prec)
    spec = np.zeros((64, 64, 33), dtype=np.complex128)
    spec[0, 0, 0] = 1000.0
    out = f.backward(spec)
    assert np.abs(out - 1000.0 / 64 ** 3).max() <= 1e-6


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_round_trip_kat(prec):
    f = ob.B200Fft((32, 32, 32), precision=prec)
    x = (np.arange(32 ** 3) % 2).astype(np.float64).reshape(32, 32, 32)
    assert np.abs(f.backward(f.forward(x)) - x).max() <= 1e-5


SHAPES = [(8, 8, 8), (16, 16, 16), (32, 32, 32), (64, 32, 16), (16, 64, 128), (48, 48, 48),
          (80, 80, 80), (96, 96, 96), (32, 40, 24), (128, 128, 128), (256, 64, 64), (4, 2, 8),
          (2, 1, 4), (512, 16, 8), (1024, 8, 4), (8, 1024, 4), (4, 8, 1024)]


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
@pytest.mark.parametrize("n", SHAPES)
def test_forward_backward_vs_oracle(oracle, prec, n):
    rng = np.random.default_rng(sum(n))
    x = rng.standard_normal((n[2], n[1], n[0]))
    f = ob.B200Fft(n, precision=prec)
    X = f.forward(x)
    Xo = oracle.r2c(x)
    assert _rel(X, Xo) <= TOL[prec] * np.log2(max(x.size, 2))
    y = f.backward(Xo)
    yo = oracle.c2r(Xo, n[0])
    assert _rel(y, yo) <= TOL[prec] * np.log2(max(x.size, 2))


def test_device_buffers_and_dtype_mix(oracle):
    import torch
    n = (32, 16, 8)
    x = np.random.default_rng(3).standard_normal((n[2], n[1], n[0]))
    f = ob.B200Fft(n, precision=ob.FP64)
    xd = torch.tensor(x, device="cuda")
    Xd = torch.zeros((n[2], n[1], n[0] // 2 + 1, 2), dtype=torch.float64, device="cuda")
    f.forward(xd, Xd)
    X = Xd.cpu().numpy()
    X = X[..., 0] + 1j * X[..., 1]
    assert _rel(X, oracle.r2c(x)) <= 1e-12
    # FP32 host buffers into an FP64 handle are converted, not rejected
    x32 = x.astype(np.float32)
    out = f.forward(x32, np.zeros((n[2], n[1], n[0] // 2 + 1), dtype=np.complex64))
    assert _rel(out, oracle.r2c(x32.astype(np.float64))) <= 1e-6


def test_size_contract_raises():
    f = ob.B200Fft((16, 16, 16), precision=ob.FP64)
    with pytest.raises(ValueError):
        f.forward(np.zeros((16, 16, 15)))
    with pytest.raises(ValueError):
        f.backward(np.zeros((16, 16, 8), dtype=np.complex128))
