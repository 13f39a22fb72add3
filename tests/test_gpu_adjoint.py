"""Hand-written adjoint of the plain PFC step vs FP64 central finite differences.

Loss L = 1/2 sum_x (psi_T - psi*)^2 after n steps; gradients with respect to r,
n0 (psi0 = n0 + fixed noise) and psi0 (checked along a random direction).
The 128^3 case is the adjoint-calibration configuration: target from
r* = -0.22, n0* = -0.28 (seed 3, 200 steps), gradients at r = -0.25,
n0 = -0.285, snapshots every 20 steps, FD with h = 1e-6 in FP64; FP32 adjoint
within 1e-4 relative.
"""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3
DT = 0.5


def run(n, psi0, r, steps, prec=ob.FP64):
    m = ob.PfcB200(n, PI4, r=r, precision=prec)
    m.initialize(DT)
    m.set_psi(psi0)
    m.step(steps)
    m.sync()
    return m.get_psi()


def loss(n, psi0, r, steps, target):
    d = run(n, psi0, r, steps) - target
    return 0.5 * float(np.dot(d.ravel(), d.ravel()))


def adjoint(n, psi0, r, steps, K, target, prec):
    m = ob.PfcB200(n, PI4, r=r, precision=prec)
    m.initialize(DT)
    m.set_psi(psi0)
    m.forward_checkpointed(steps, K)
    psiT = m.get_psi()
    g, gr, gn = m.adjoint(psiT - target)
    return g, gr, gn


def check(n, steps, K, r, n0, rs, n0s, seed, prec, tol, h=1e-6):
    target = run(n, ob.ic_noise(n, n0s, 0.01, seed), rs, steps)
    psi0 = ob.ic_noise(n, n0, 0.01, seed)
    g, gr, gn = adjoint(n, psi0, r, steps, K, target, prec)
    fd_r = (loss(n, psi0, r + h, steps, target) - loss(n, psi0, r - h, steps, target)) / (2 * h)
    fd_n0 = (loss(n, psi0 + h, r, steps, target) - loss(n, psi0 - h, r, steps, target)) / (2 * h)
    v = np.random.default_rng(seed + 1).standard_normal(psi0.shape)
    v /= np.linalg.norm(v)
    fd_v = (loss(n, psi0 + h * v, r, steps, target) - loss(n, psi0 - h * v, r, steps, target)) / (2 * h)
    assert abs(gr - fd_r) <= tol * abs(fd_r), (gr, fd_r)
    assert abs(gn - fd_n0) <= tol * abs(fd_n0), (gn, fd_n0)
    gv = float(np.dot(g.ravel(), v.ravel()))
    assert abs(gv - fd_v) <= tol * max(abs(fd_v), 1e-3 * np.linalg.norm(g)), (gv, fd_v)
    return g, gr, gn


def test_adjoint_fp64_small():
    check((32, 32, 32), 30, 7, -0.25, -0.285, -0.22, -0.28, 11, ob.FP64, 1e-6)


def test_adjoint_calibration_128_fp32():
    n = (128, 128, 128)
    g32, gr32, gn32 = check(n, 200, 20, -0.25, -0.285, -0.22, -0.28, 3, ob.FP32, 1e-4)
    # FP32 adjoint against the FP64 adjoint of the same problem
    target = run(n, ob.ic_noise(n, -0.28, 0.01, 3), -0.22, 200)
    g64, gr64, gn64 = adjoint(n, ob.ic_noise(n, -0.285, 0.01, 3), -0.25, 200, 20, target, ob.FP64)
    assert abs(gr32 - gr64) <= 1e-4 * abs(gr64)
    assert abs(gn32 - gn64) <= 1e-4 * abs(gn64)
    assert np.linalg.norm((g32 - g64).ravel()) <= 1e-4 * np.linalg.norm(g64.ravel())


def test_autograd_function_matches_adjoint():
    import torch
    from openpfc_b200.autograd import PfcEvolve, make_model
    n = (32, 32, 32)
    target = torch.tensor(run(n, ob.ic_noise(n, -0.28, 0.01, 5), -0.22, 20), device="cuda")
    psi0 = torch.tensor(ob.ic_noise(n, -0.285, 0.01, 5), device="cuda", requires_grad=True)
    r = torch.tensor(-0.25, dtype=torch.float64, requires_grad=True)
    model = make_model(n, PI4, precision=ob.FP64, dt=DT)
    psiT = PfcEvolve.apply(psi0, r, model, 20, 5)
    L = 0.5 * ((psiT - target) ** 2).sum()
    L.backward()
    g, gr, _ = adjoint(n, psi0.detach().cpu().numpy(), -0.25, 20, 5, target.cpu().numpy(), ob.FP64)
    np.testing.assert_allclose(psi0.grad.cpu().numpy(), g, rtol=1e-10, atol=1e-14)
    assert abs(float(r.grad) - gr) <= 1e-10 * abs(gr)
