"""The sharded single-field FFT and PFC step (z slabs for the x and y passes,
kx slabs for the z transform and update, all-to-all transposes between them)
with P ranks emulated on one GPU, against the FP64 oracle of the whole field.
Tolerances as for one handle: FP64 <= 1e-11 (steps) / 1e-12 (transforms), FP32
<= 1e-5 relative L2."""
import math

import numpy as np
import pytest

import openpfc_b200 as ob
from openpfc_b200.sharded import LocalComm, ShardedFft, ShardedPfc

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def slabs(field, P):
    n2loc = field.shape[0] // P
    return [field[q * n2loc:(q + 1) * n2loc] for q in range(P)]


@pytest.mark.parametrize("P", [1, 2, 4])
@pytest.mark.parametrize("n", [(32, 16, 64), (64, 32, 32)])
def test_sharded_fft_vs_oracle(oracle, P, n):
    x = np.random.default_rng(5).standard_normal((n[2], n[1], n[0]))
    f = ShardedFft(n, LocalComm(P), precision=ob.FP64)
    spec = f.forward(slabs(x, P))
    whole = np.concatenate(spec, axis=2)  # kx slabs side by side: (N2, N1, N0/2 + 1)
    ref = oracle.r2c(x)
    assert np.abs(whole - ref).max() <= 1e-12 * np.abs(ref).max()
    back = np.concatenate(f.backward(spec), axis=0)
    assert np.abs(back - x).max() <= 1e-12 * np.abs(x).max()
    f.close()


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("P", [1, 2, 4])
def test_sharded_plain_step_vs_oracle(oracle, prec, tol, P):
    n = (64, 64, 64)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 42)
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 12)
    m = ShardedPfc(n, PI4, LocalComm(P), r=-0.25, precision=prec)
    m.initialize(0.5)
    m.set_psi(slabs(psi0, P))
    m.step(5)
    mid = np.concatenate(m.get_psi(), axis=0)  # output mid-run, then carry on
    assert rel_l2(mid, oracle.run_plain(psi0, PI4, -0.25, 0.5, 5)) <= tol
    m.step(7)
    got = np.concatenate(m.get_psi(), axis=0)
    assert rel_l2(got, ref) <= tol
    assert abs(got.mean() - psi0.mean()) <= 1e-6
    m.close()


@pytest.mark.parametrize("P", [2, 4])
def test_sharded_filtered_step_vs_oracle(oracle, P):
    n = (64, 32, 32)
    psi0 = oracle.ic_seeds(n, PI4, -0.10, 0.001, 2, 8.0, 0.2, 4)
    ref = oracle.run_filtered(psi0, PI4, -0.3, 0.5, -0.1, -0.5, 0.3, 0.5, 8)
    m = ShardedPfc(n, PI4, LocalComm(P), r=-0.3, precision=ob.FP64, model="filtered")
    m.initialize(0.5)
    m.set_psi(slabs(psi0, P))
    m.step(8)
    assert rel_l2(np.concatenate(m.get_psi(), axis=0), ref) <= 1e-11
    m.close()


def test_sharded_sizes_are_checked():
    with pytest.raises(ValueError):
        ShardedPfc((64, 32, 30), PI4, LocalComm(4))
