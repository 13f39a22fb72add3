"""Hand-written adjoint of the filtered, Tungsten and Aluminum steps against
FP64 central finite differences, through the C ABI.

The adjoint step applies the conjugate spectral multiplies (opL, opN), the
adjoint of the mean-field filter (the filter itself: chi is real and even) and
the Jacobian of the model's nonlinearity -- p2 v + p3 v^2 + p4 v^3 of the
filtered density for the filtered model; 2 p3b u + 3 p4b u^2 - stabP and
2 q3b v + 3 q4b v^2 of psi and psi_MF for the Tungsten form.  Loss
L = 1/2 sum_x (psi_T - psi*)^2; gradients with respect to n0 (psi0 shifted
uniformly), r (filtered model) and psi0 along a random direction.  FD in FP64
with h = 1e-6; FP64 adjoint within 1e-6 relative, FP32 adjoint within 1e-4.
"""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3


def filtered(n, r, prec):
    m = ob.FilteredB200(n, PI4, r=r, alpha=0.5, p2=-0.1, p3=-0.5, p4=0.3, precision=prec)
    m.initialize(0.5)
    return m


def tungsten(n, r, prec):
    dx = 1.1107207345395915
    m = ob.TungstenB200(n, [dx] * 3, precision=prec)
    m.initialize(1.0)
    return m


def aluminum(n, r, prec):
    from test_gpu_aluminum import params
    m = ob.AluminumB200(n, [1.0] * 3, params(), precision=prec)
    m.initialize(1e-2)
    return m


def final(make, n, psi0, r, steps, prec=ob.FP64):
    m = make(n, r, prec)
    m.set_psi(psi0)
    m.step(steps)
    m.sync()
    return m.get_psi()


def loss(make, n, psi0, r, steps, target):
    d = final(make, n, psi0, r, steps) - target
    return 0.5 * float(np.dot(d.ravel(), d.ravel()))


def check(make, n, psi0, target, r, steps, K, prec, tol, has_r, h=1e-6, seed=1):
    m = make(n, r, prec)
    m.set_psi(psi0)
    m.forward_checkpointed(steps, K)
    g, gr, gn = m.adjoint(m.get_psi() - target)
    fd_n0 = (loss(make, n, psi0 + h, r, steps, target) - loss(make, n, psi0 - h, r, steps, target)) / (2 * h)
    assert abs(gn - fd_n0) <= tol * abs(fd_n0), (gn, fd_n0)
    v = np.random.default_rng(seed).standard_normal(psi0.shape)
    v /= np.linalg.norm(v)
    fd_v = (loss(make, n, psi0 + h * v, r, steps, target) - loss(make, n, psi0 - h * v, r, steps, target)) / (2 * h)
    gv = float(np.dot(g.ravel(), v.ravel()))
    assert abs(gv - fd_v) <= tol * max(abs(fd_v), 1e-3 * np.linalg.norm(g)), (gv, fd_v)
    if has_r:
        fd_r = (loss(make, n, psi0, r + h, steps, target) - loss(make, n, psi0, r - h, steps, target)) / (2 * h)
        assert abs(gr - fd_r) <= tol * abs(fd_r), (gr, fd_r)
    else:
        assert math.isnan(gr)  # r is not a parameter of the model
    return g


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-6), (ob.FP32, 1e-4)])
def test_filtered_adjoint_vs_fd(prec, tol):
    n = (32, 32, 32)
    target = final(filtered, n, ob.ic_seeds(n, PI4, -0.12, 0.01, 3, 8.0, 0.2, 5), -0.28, 16)
    psi0 = ob.ic_seeds(n, PI4, -0.10, 0.01, 3, 8.0, 0.2, 5)
    check(filtered, n, psi0, target, -0.3, 16, 5, prec, tol, has_r=True)


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-6), (ob.FP32, 1e-4)])
def test_tungsten_adjoint_vs_fd(oracle, prec, tol):
    n = (32, 32, 32)
    dx = 1.1107207345395915
    origin = [-0.5 * dx * 32] * 3
    base = oracle.ic_seed_inside(np.full((32, 32, 32), -0.4), [dx] * 3, origin, 12.0, -0.047, 0.215936)
    noise = ob.ic_noise(n, 0.0, 0.01, 9)
    target = final(tungsten, n, base + 0.005, 0.0, 8)
    check(tungsten, n, base + noise, target, 0.0, 8, 3, prec, tol, has_r=False)


def test_aluminum_adjoint_vs_fd():
    from test_gpu_aluminum import ic
    n = (32, 32, 32)
    psi0 = ic()
    target = final(aluminum, n, psi0 + 0.002, 0.0, 6)
    check(aluminum, n, psi0, target, 0.0, 6, 2, ob.FP64, 1e-6, has_r=False)


def test_filtered_adjoint_fp32_matches_fp64_64():
    n = (64, 64, 64)
    target = final(filtered, n, ob.ic_seeds(n, PI4, -0.12, 0.01, 3, 10.0, 0.2, 7), -0.28, 30)
    psi0 = ob.ic_seeds(n, PI4, -0.10, 0.01, 3, 10.0, 0.2, 7)
    out = {}
    for prec in (ob.FP32, ob.FP64):
        m = filtered(n, -0.3, prec)
        m.set_psi(psi0)
        m.forward_checkpointed(30, 10)
        out[prec] = m.adjoint(m.get_psi() - target)
    (g32, r32, n32), (g64, r64, n64) = out[ob.FP32], out[ob.FP64]
    assert abs(r32 - r64) <= 1e-4 * abs(r64)
    assert abs(n32 - n64) <= 1e-4 * abs(n64)
    assert np.linalg.norm((g32 - g64).ravel()) <= 1e-4 * np.linalg.norm(g64.ravel())


def test_autograd_harness_filtered():
    import torch
    from openpfc_b200.autograd import PfcEvolve
    n = (32, 32, 32)
    target = torch.tensor(final(filtered, n, ob.ic_seeds(n, PI4, -0.12, 0.01, 2, 8.0, 0.2, 3), -0.28, 10),
                          device="cuda")
    psi0_np = ob.ic_seeds(n, PI4, -0.10, 0.01, 2, 8.0, 0.2, 3)
    psi0 = torch.tensor(psi0_np, device="cuda", requires_grad=True)
    r = torch.tensor(-0.3, dtype=torch.float64, requires_grad=True)
    model = filtered(n, -0.3, ob.FP64)
    L = 0.5 * ((PfcEvolve.apply(psi0, r, model, 10, 4) - target) ** 2).sum()
    L.backward()
    m = filtered(n, -0.3, ob.FP64)
    m.set_psi(psi0_np)
    m.forward_checkpointed(10, 4)
    g, gr, _ = m.adjoint(m.get_psi() - target.cpu().numpy())
    np.testing.assert_allclose(psi0.grad.cpu().numpy(), g, rtol=1e-10, atol=1e-14)
    assert abs(float(r.grad) - gr) <= 1e-10 * abs(gr)
