"""Caller-supplied ETD1 operators (OPFC_MODEL_USER_ETD, the GPU backend of the
reference's Etd1Stepper, include/openpfc/kernel/simulation/steppers/etd1.hpp):
the plain PFC operators fed through it reproduce the oracle's plain step; pure
diffusion reproduces the exact Fourier-mode decay; non-conserving k = 0
entries are refused."""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu
PI4 = [math.pi / 4] * 3


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
def test_user_etd_reproduces_plain_pfc(oracle, prec, tol):
    n = (64, 48, 32)
    opL, opN = oracle.ops_plain(n, PI4, -0.25, 0.5)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 9)
    m = ob.EtdB200(n, PI4, p3=3.0, precision=prec)  # N = p3 v^3 / 3 = psi^3, chi = 1
    m.set_operators(opL, opN)
    m.initialize(0.5)
    m.set_psi(psi0)
    m.step(10)
    m.sync()
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 10)
    assert np.linalg.norm((m.get_psi() - ref).ravel()) <= tol * np.linalg.norm(ref.ravel())


def test_user_etd_diffusion_exact():
    n = (32, 32, 32)
    dx, D, dt, steps = [0.5] * 3, 0.7, 0.05, 12
    k = [2 * np.pi * np.fft.fftfreq(n[a], d=dx[a]) for a in range(3)]
    kx = 2 * np.pi * np.fft.rfftfreq(n[0], d=dx[0])
    k2 = kx[None, None, :] ** 2 + k[1][None, :, None] ** 2 + k[2][:, None, None] ** 2
    eL = np.exp(-D * k2 * dt)
    psi0 = np.random.default_rng(4).standard_normal((n[2], n[1], n[0])) * 0.1 + 0.3
    m = ob.EtdB200(n, dx)  # N = 0: heat equation
    m.set_operators(eL, np.zeros_like(eL))
    m.initialize(dt)
    m.set_psi(psi0)
    m.step(steps)
    m.sync()
    exact = np.fft.irfftn(np.fft.rfftn(psi0) * np.exp(-D * k2 * dt * steps), s=psi0.shape)
    assert np.abs(m.get_psi() - exact).max() <= 1e-12


def test_user_etd_refuses_non_conserving_operators():
    n = (16, 16, 16)
    shape = (n[2], n[1], n[0] // 2 + 1)
    m = ob.EtdB200(n, [1.0] * 3)
    bad = np.ones(shape)
    bad.flat[0] = 0.9
    with pytest.raises(ob.OpfcError):
        m.set_operators(bad, np.zeros(shape))
    with pytest.raises(ob.OpfcError):
        m.initialize(0.1)  # no operators yet
