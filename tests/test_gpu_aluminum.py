"""Aluminum PFC variant on the GPU against the oracle and the reference
test's golden norms (apps/aluminumNew/aluminumTest.cpp:83-110: 32^3, dx 1,
dt 1e-2, SeedGridFCC rseed 42; sum psi^2 before each of 5 steps, +-0.1)."""
import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu
NORMS = [1297.08, 1250.21, 1209.28, 1173.19, 1141.09]


def params():
    p = ob.AluminumParams()
    p.T0 = 1.0
    for k, v in dict(n0=-0.0060, alpha=0.20, n_sol=-0.036, n_vap=-1.297, T_const=980, T_min=780, T_max=1280,
                     T0=89285.0, Bx=0.817900686921996, G_grid=0, V_grid=0, x_initial=130, alpha_farTol=0.001,
                     lambda_=0.22, stabP=0.0, shift_u=1.0, shift_s=0.0, p2_bar=0.8286531831,
                     p3_bar=-0.04204863, p4_bar=0.007533, q20_bar=0.016531729105214, q21_bar=5.467,
                     q30_bar=1.7152418049986, q31_bar=0.45, q40_bar=0.787482).items():
        setattr(p, k, v)
    return p


def ic():
    return ob.ic_seed_grid_fcc(np.full((32, 32, 32), -0.0060), [1.0] * 3, [0.0] * 3, 1, 2, 2, 8.0, 4.0, 0.4,
                               -0.036, 42)


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
def test_aluminum_golden_norms_and_oracle(oracle, prec, tol):
    psi0 = ic()
    m = ob.AluminumB200((32, 32, 32), [1.0] * 3, params(), precision=prec)
    m.initialize(1e-2)
    m.set_psi(psi0)
    norms = [float((psi0 ** 2).sum())]
    for _ in range(4):
        m.step(1)
        m.sync()
        norms.append(float((m.get_psi() ** 2).sum()))
    np.testing.assert_allclose(norms, NORMS, atol=0.1, rtol=0)
    op = oracle.AluminumParams.test_case()
    ref = oracle.run_aluminum(psi0, [1.0] * 3, [0.0] * 3, op, 1e-2, 4, t0=1.0)
    got = m.get_psi()
    assert np.linalg.norm((got - ref).ravel()) <= tol * np.linalg.norm(ref.ravel())
    mf = m.get_psi_mf()
    assert np.isfinite(mf).all() and abs(mf.mean() - got.mean()) <= 1e-6


def test_aluminum_larger_grid_vs_oracle(oracle):
    n = (64, 48, 32)
    psi0 = ob.ic_seed_grid_fcc(np.full(n[::-1], -0.0060), [1.0] * 3, [0.0] * 3, 1, 2, 2, 10.0, 6.0, 0.4, -0.036, 3)
    p = params()
    p.q4_bar, p.stabP, p.q2_bar_L = 0.3, 0.1, 0.2
    op = oracle.AluminumParams.test_case()
    op.q4_bar, op.stabP, op.q2_bar_L = 0.3, 0.1, 0.2
    m = ob.AluminumB200(n, [1.0] * 3, p, precision=ob.FP64)
    m.initialize(1e-2)
    m.set_psi(psi0)
    m.step(6)
    m.sync()
    ref = oracle.run_aluminum(psi0, [1.0] * 3, [0.0] * 3, op, 1e-2, 6)
    assert np.linalg.norm((m.get_psi() - ref).ravel()) <= 1e-11 * np.linalg.norm(ref.ravel())


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
def test_aluminum_moving_gradient_vs_oracle(oracle, prec, tol):
    # G_grid != 0: T_var(x, t) = G (dist - x_initial - V t) with the wrap at
    # m_xpos, a third field P*psi, time t0 + s dt for step s (Aluminum.hpp:262-307)
    vals = dict(G_grid=2.0, V_grid=0.5, q4_bar=0.787482, tau_const=0.3, m_xpos=5.0, x_initial=4.0, stabP=0.05)
    p, op = params(), oracle.AluminumParams.test_case()
    for k, v in vals.items():
        setattr(p, k, v)
        setattr(op, k, v)
    origin = [-3.0, 0.0, 0.0]
    psi0 = ic()
    m = ob.AluminumB200((32, 32, 32), [1.0] * 3, p, precision=prec, origin=origin)
    m.initialize(1e-2)
    m.set_psi(psi0)
    m.set_time(0.3, 1e-2)
    m.step(4)
    m.sync()
    ref = oracle.run_aluminum(psi0, [1.0] * 3, origin, op, 1e-2, 4, t0=0.3, dt_t=1e-2)
    got = m.get_psi()
    assert np.linalg.norm((got - ref).ravel()) <= tol * np.linalg.norm(ref.ravel())
    # the gradient acts: without it the result differs
    base = oracle.run_aluminum(psi0, [1.0] * 3, origin, oracle.AluminumParams.test_case(), 1e-2, 4, t0=0.3)
    assert np.abs(ref - base).max() > 1e-6
