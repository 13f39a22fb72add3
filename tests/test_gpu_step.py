"""GPU parity of the PFC time step against the FP64 oracle, through the C ABI.

Tolerances follow the target: relative L2 <= 1e-11 in FP64 and <= 1e-5 in FP32
after 100 steps (rel-L2 = ||psi - psi_ref||_2 / ||psi_ref||_2 over all cells).
The Tungsten regression norms are the reference's own golden values
(apps/tungsten/tests/test_tungsten.cpp:288-300, tolerance 0.1 absolute).
"""
import json
import math
import os

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def run_plain(n, prec, psi0, steps, r=-0.25, dt=0.5, dx=PI4):
    m = ob.PfcB200(n, dx, r=r, precision=prec)
    m.initialize(dt)
    m.set_psi(psi0)
    m.step(steps)
    m.sync()
    return m, m.get_psi()


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
def test_plain_config1_64cubed_100_steps(oracle, prec, tol):
    # config: 64^3, dx = pi/4, dt = 0.5, r = -0.25, psi0 = -0.285 + U(-0.01, 0.01), seed 42
    n = (64, 64, 64)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 42)
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 100)
    m, psi = run_plain(n, prec, psi0, 100)
    assert rel_l2(psi, ref) <= tol
    # mass (k = 0 mode carried in FP64) is exactly the initial mean
    assert abs(m.mass() - oracle.compensated_sum(psi0) / psi0.size) <= 1e-15
    assert abs(m.mass() - ref.mean()) <= 1e-12
    if prec == ob.FP64:
        f_gpu = m.free_energy()
        f_ref = oracle.free_energy_plain(ref, PI4, -0.25)
        assert abs(f_gpu - f_ref) <= 1e-10 * abs(f_ref)


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("n", [(32, 32, 32), (16, 32, 64), (48, 48, 48), (128, 64, 32)])
def test_plain_shapes(oracle, prec, tol, n):
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 7)
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 20)
    _, psi = run_plain(n, prec, psi0, 20)
    assert rel_l2(psi, ref) <= tol


def test_psi_hat_matches_oracle_transform(oracle):
    n = (32, 32, 32)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 11)
    m, psi = run_plain(n, ob.FP64, psi0, 10)
    ph = m.get_psi_hat()
    ref = oracle.r2c(psi)
    assert np.abs(ph - ref).max() <= 1e-9 * np.abs(ref).max()


def _tungsten_ic(oracle, n=32):
    dx = 1.1107207345395915
    origin = [-0.5 * dx * n] * 3
    psi = np.full((n, n, n), -0.4)
    return oracle.ic_seed_inside(psi, [dx] * 3, origin, 18.0, -0.047, 0.215936), dx


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_tungsten_golden_norms(oracle, golden_dir, prec):
    g = json.load(open(os.path.join(golden_dir, "tungsten_norms_32.json")))
    psi0, dx = _tungsten_ic(oracle)
    m = ob.TungstenB200((32, 32, 32), [dx] * 3, precision=prec)
    m.initialize(g["dt"])
    m.set_psi(psi0)
    norms = []
    for _ in range(10):
        m.step(1)
        m.sync()
        norms.append(float((m.get_psi() ** 2).sum()))
    np.testing.assert_allclose(norms, g["norms"][1:], atol=g["abs_tol"], rtol=0)
    if prec == ob.FP64:
        np.testing.assert_allclose(norms, g["norms"][1:], rtol=1e-10)


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
def test_tungsten_vs_oracle_and_psi_mf(oracle, prec, tol):
    psi0, dx = _tungsten_ic(oracle)
    p = oracle.TungstenParams.defaults()
    ref = oracle.run_tungsten(psi0, [dx] * 3, p, 1.0, 10)
    m = ob.TungstenB200((32, 32, 32), [dx] * 3, precision=prec)
    m.initialize(1.0)
    m.set_psi(psi0)
    m.step(10)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= tol
    # psi_MF = F^-1[filterMF F[psi]]
    ops = oracle.ops_tungsten((32, 32, 32), [dx] * 3, p, 1.0)
    mf_ref = oracle.c2r(oracle.r2c(ref) * ops["filterMF"], 32)
    assert rel_l2(m.get_psi_mf(), mf_ref) <= tol


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
def test_filtered_vs_oracle(oracle, prec, tol):
    n = (64, 64, 64)
    psi0 = oracle.ic_seeds(n, PI4, -0.10, 0.001, 3, 10.0, 0.2, 9)
    ref = oracle.run_filtered(psi0, PI4, -0.3, 0.5, -0.1, -0.5, 0.3, 0.5, 30)
    m = ob.FilteredB200(n, PI4, precision=prec)
    m.initialize(0.5)
    m.set_psi(psi0)
    m.step(30)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= tol


def test_device_resident_io(oracle):
    import torch
    n = (32, 32, 32)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 5)
    m = ob.PfcB200(n, PI4, precision=ob.FP32)
    m.initialize(0.5)
    m.set_psi(torch.tensor(psi0, dtype=torch.float32, device="cuda"))
    m.step(5)
    out = torch.zeros(n[::-1], dtype=torch.float32, device="cuda")
    m.get_psi(out)
    ref = oracle.run_plain(psi0.astype(np.float32).astype(np.float64), PI4, -0.25, 0.5, 5)
    assert rel_l2(out.cpu().numpy().astype(np.float64), ref) <= 1e-5


def test_nonfinite_is_reported():
    n = (16, 16, 16)
    m = ob.PfcB200(n, PI4, precision=ob.FP32)
    m.initialize(0.5)
    psi = np.full(n, -0.285)
    psi[3, 4, 5] = 1e20  # psi^3 overflows FP32
    m.set_psi(psi)
    m.step(1)
    with pytest.raises(ob.OpfcError) as e:
        m.sync()
    assert e.value.status == -4


def test_call_order_errors():
    m = ob.PfcB200((16, 16, 16), PI4)
    with pytest.raises(ob.OpfcError):
        m.step(1)  # before initialize
    m.initialize(0.5)
    with pytest.raises(ob.OpfcError):
        m.step(1)  # before set_psi
    with pytest.raises(ValueError):
        m.set_psi(np.zeros((16, 16, 8)))


def test_nvtx_eager_steps_match_oracle(oracle, monkeypatch):
    """OPFC_NVTX=1: steps run eagerly inside NVTX ranges named after the
    reference's regions, with the same results as the graph path."""
    monkeypatch.setenv("OPFC_NVTX", "1")
    n = (32, 32, 32)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 17)
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 6)
    _, psi = run_plain(n, ob.FP64, psi0, 6)
    assert rel_l2(psi, ref) <= 1e-11
