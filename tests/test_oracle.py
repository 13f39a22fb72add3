"""CPU tests that pin the FP64 oracle to the reference's own known answers.

The oracle is the checker for every GPU parity test, so it is pinned first:
FFT conventions (tests/unit/kernel/fft/test_fft.cpp, tests/unit/runtime/gpu/
test_fft_cuda.cpp), ETD coefficients (tests/unit/kernel/integrator/
test_spectral_exp_coefficients.cpp), the reference's own Tungsten operator tables
(tests/golden/tungsten_ops_16x12x10.npz, produced by the reference headers) and
the Tungsten golden norms (apps/tungsten/tests/test_tungsten.cpp:288-300).
"""
import json
import math
import os

import numpy as np
import pytest

from oracle.oracle import reference_dir as _reference_dir


@pytest.mark.parametrize("shape", [(8, 8, 8), (10, 12, 16), (8, 5, 6), (32, 32, 32), (5, 3, 2),
                                   (1, 1, 8), (1, 1, 2), (6, 10, 48), (4, 4, 80)])
def test_r2c_c2r_match_numpy(oracle, shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape)
    X = oracle.r2c(a)
    Y = np.fft.rfftn(a)
    assert np.abs(X - Y).max() <= 1e-13 * np.abs(Y).max()
    back = oracle.c2r(X, shape[2])
    assert np.abs(back - a).max() <= 1e-13


def test_fft_forward_dc_kat(oracle):
    # tests/unit/kernel/fft/test_fft.cpp:28-47
    x = np.array([0.000, 0.785, 1.571, 2.356, 3.142, 3.927, 4.712, 5.498]).reshape(1, 1, 8)
    assert abs(oracle.r2c(x)[0, 0, 0].real - 21.991) <= 0.01


def test_fft_backward_normalisation_kat(oracle):
    # tests/unit/kernel/fft/test_fft.cpp:50-70: 1/N on backward
    out = oracle.c2r(np.array([1 + 0j, 2 + 0j]).reshape(1, 1, 2), 2)
    assert abs(out[0, 0, 0] - 1.5) <= 0.01


def test_fft_dc_only_backward_kat(oracle):
    # tests/unit/runtime/gpu/test_fft_cuda.cpp:84-130
    spec = np.zeros((64, 64, 33), dtype=np.complex128)
    spec[0, 0, 0] = 1000.0
    out = oracle.c2r(spec, 64)
    assert np.abs(out - 1000.0 / 64 ** 3).max() <= 1e-6


def test_fft_round_trip_kat(oracle):
    # tests/unit/runtime/gpu/test_fft_cuda.cpp:138-189 (alternating 0, 1)
    x = (np.arange(32 ** 3) % 2).astype(np.float64).reshape(32, 32, 32)
    assert np.abs(oracle.c2r(oracle.r2c(x), 32) - x).max() <= 1e-5


@pytest.mark.parametrize("L,dt", [(-4.0, 0.25), (1.5, 0.25), (-2.0, 0.0)])
def test_spectral_exp_nonzero(oracle, L, dt):
    # test_spectral_exp_coefficients.cpp:29-58
    e, p = oracle.spectral_exp(L, dt)
    assert e == pytest.approx(math.exp(L * dt), rel=1e-14, abs=1e-15)
    ref = math.expm1(L * dt) / L if dt != 0 else 0.0
    assert p == pytest.approx(ref, rel=1e-14, abs=1e-15)


def test_spectral_exp_taylor(oracle):
    # test_spectral_exp_coefficients.cpp:60-87
    dt = 0.1
    e, p = oracle.spectral_exp(0.0, dt)
    assert abs(e - 1.0) <= 1e-15 and abs(p - dt) <= 1e-15
    e, p = oracle.spectral_exp(1e-13, dt)
    assert abs(p - (dt + 0.5 * 1e-13 * dt * dt)) <= 1e-18
    e, p = oracle.spectral_exp(1e-12, dt)
    assert p == pytest.approx(math.expm1(1e-12 * dt) / 1e-12, rel=1e-12)


def test_mt19937_64_known_value(oracle):
    # the C++ standard's check value for the 10000th draw of mt19937_64(5489)
    assert int(oracle.mt64_stream(5489, 10000)[-1]) == 9981545732273789042


def test_tungsten_derived_params_match_reference(oracle, golden_dir):
    g = np.load(os.path.join(golden_dir, "tungsten_ops_16x12x10.npz"))
    d = oracle.tungsten_derived(oracle.TungstenParams.defaults())
    mine = [d.tau, d.p2b, d.p3b, d.p4b, d.q20b, d.q21b, d.q30b, d.q31b, d.q40b, d.q2b, d.q3b, d.q4b]
    np.testing.assert_allclose(mine, g["derived"], rtol=1e-15, atol=0)


def test_tungsten_tables_match_reference(oracle, golden_dir):
    g = np.load(os.path.join(golden_dir, "tungsten_ops_16x12x10.npz"))
    ops = oracle.ops_tungsten(tuple(g["n"]), [float(g["dx"])] * 3, oracle.TungstenParams.defaults(),
                              float(g["dt"]))
    for k in ("filterMF", "exp_Ldt", "n_weight"):
        np.testing.assert_allclose(ops[k], g[k], rtol=1e-14, atol=1e-300, err_msg=k)


@pytest.mark.skipif(_reference_dir() is None, reason="reference tree absent (OPENPFC_REFERENCE_DIR)")
def test_tungsten_tables_match_reference_live(oracle, tmp_path):
    oracle.build(ref=True)
    n, dx, dt = (8, 10, 12), 0.9, 0.5
    r = oracle.ref_ops(n, dx, dt, str(tmp_path))
    ops = oracle.ops_tungsten(n, [dx] * 3, oracle.TungstenParams.defaults(), dt)
    for k in ("filterMF", "exp_Ldt", "n_weight"):
        np.testing.assert_allclose(ops[k], r[k], rtol=1e-14, atol=1e-300, err_msg=k)


def _tungsten_ic(oracle, n=32):
    dx = 1.1107207345395915
    origin = [-0.5 * dx * n] * 3
    psi = np.full((n, n, n), -0.4)
    return oracle.ic_seed_inside(psi, [dx] * 3, origin, 18.0, -0.047, 0.215936), dx


def test_tungsten_golden_norms(oracle, golden_dir):
    g = json.load(open(os.path.join(golden_dir, "tungsten_norms_32.json")))
    psi, dx = _tungsten_ic(oracle)
    assert abs(float((psi ** 2).sum()) - g["norms"][0]) <= g["abs_tol"]
    _, norms = oracle.run_tungsten(psi, [dx] * 3, oracle.TungstenParams.defaults(), g["dt"], 10,
                                   norms=True)
    # reference tolerance is 0.1 absolute; the restatement agrees far tighter
    np.testing.assert_allclose(norms, g["norms"][1:], atol=g["abs_tol"], rtol=0)
    np.testing.assert_allclose(norms, g["norms"][1:], rtol=1e-11)


def test_plain_mass_conserved_and_energy_decreases(oracle):
    # conserved dynamics (the precedent: tests/integration/scenarios/
    # complete_simulation/test_mass_conservation.cpp:15-48, drift <= 1e-12)
    n, dx, r, dt = (16, 16, 16), [math.pi / 4] * 3, -0.25, 0.5
    psi = oracle.ic_noise(n, -0.285, 0.01, 42)
    m0 = psi.mean()
    f_prev = oracle.free_energy_plain(psi, dx, r)
    for _ in range(5):
        psi = oracle.run_plain(psi, dx, r, dt, 4)
        assert abs(psi.mean() - m0) <= 1e-12
        f = oracle.free_energy_plain(psi, dx, r)
        assert f <= f_prev + 1e-9
        f_prev = f


def test_filtered_step_runs_and_conserves(oracle):
    n, dx = (16, 16, 16), [math.pi / 4] * 3
    psi = oracle.ic_seeds(n, dx, -0.10, 0.001, 2, 4.0, 0.2, 5)
    m0 = psi.mean()
    out = oracle.run_filtered(psi, dx, -0.3, 0.5, -0.1, -0.5, 0.3, 0.5, 5)
    assert np.isfinite(out).all()
    assert abs(out.mean() - m0) <= 1e-12


# apps/aluminumNew/aluminumTest.cpp:83-110: 32^3, dx = 1, origin 0, dt = 1e-2;
# psi = n0 everywhere, then SeedGridFCC(Nx 1, Ny 2, Nz 2, X0 8, radius 4,
# amplitude 0.4, rho -0.036, rseed 42); sum psi^2 before each of 5 steps,
# +-0.1 absolute.  Parameters the test leaves unset stay 0 (q4_bar, q2_bar_L,
# tau_const), so the moving-temperature terms vanish (G_grid = 0).
ALUMINUM_NORMS = [1297.08, 1250.21, 1209.28, 1173.19, 1141.09]


def aluminum_ic(oracle):
    psi = np.full((32, 32, 32), -0.0060)
    return oracle.ic_seed_grid_fcc(psi, [1.0] * 3, [0.0] * 3, 1, 2, 2, 8.0, 4.0, 0.4, -0.036, 42)


def test_aluminum_golden_norms(oracle):
    psi = aluminum_ic(oracle)
    assert abs(float((psi ** 2).sum()) - ALUMINUM_NORMS[0]) <= 0.1
    _, norms = oracle.run_aluminum(psi, [1.0] * 3, [0.0] * 3, oracle.AluminumParams.test_case(), 1e-2, 4,
                                   t0=1.0, norms=True)
    np.testing.assert_allclose(norms, ALUMINUM_NORMS[1:], atol=0.1, rtol=0)
    # printed to 6 significant digits in the reference: the restatement rounds to them
    np.testing.assert_allclose(norms, ALUMINUM_NORMS[1:], rtol=5e-6)


def test_aluminum_moving_gradient_conserves_mass(oracle):
    # G_grid != 0: position- and time-dependent temperature, kernel term on P*psi
    p = oracle.AluminumParams.test_case()
    p.G_grid, p.V_grid, p.q4_bar, p.tau_const = 2.0, 0.5, 0.787482, 0.3
    psi = aluminum_ic(oracle)
    out = oracle.run_aluminum(psi, [1.0] * 3, [0.0] * 3, p, 1e-2, 3, t0=0.0, dt_t=1e-2)
    assert np.isfinite(out).all()
    assert abs(out.mean() - psi.mean()) <= 1e-12
    base = oracle.run_aluminum(psi, [1.0] * 3, [0.0] * 3, oracle.AluminumParams.test_case(), 1e-2, 3)
    assert np.abs(out - base).max() > 1e-6  # the gradient terms act


RANDOM_SEEDS_CASES = {
    "n32": ((32, 32, 32), (8.0, 8.0, 8.0), (-128.0, -128.0, -128.0), 0.5, 0.2),
    "n16": ((16, 16, 16), (16.0, 16.0, 16.0), (-128.0, -128.0, -128.0), 0.65, 0.15),
}


@pytest.mark.parametrize("key", list(RANDOM_SEEDS_CASES))
def test_random_seeds_matches_reference_seed_class(oracle, golden_dir, key):
    """RandomSeeds on the domains of test_ic_random_seeds.cpp: the oracle equals,
    bit for bit, the field computed with the reference's own Seed class
    (tests/golden/random_seeds.npz), and has the properties that test checks:
    some cells inside seeds, values within density +- 12 amplitude (+0.1),
    deterministic."""
    n, dx, org, rho, amp = RANDOM_SEEDS_CASES[key]
    g = np.load(os.path.join(golden_dir, "random_seeds.npz"))[key]
    got = oracle.ic_random_seeds(n, dx, org, rho, amp)
    np.testing.assert_array_equal(got, g)
    inside = got[got != 0.0]
    assert inside.size > 0
    assert inside.min() >= rho - 12 * amp - 0.1 and inside.max() <= rho + 12 * amp + 0.1
    np.testing.assert_array_equal(oracle.ic_random_seeds(n, dx, org, rho, amp), got)


@pytest.mark.skipif(_reference_dir() is None, reason="reference tree absent (OPENPFC_REFERENCE_DIR)")
def test_random_seeds_matches_reference_live(oracle, tmp_path):
    oracle.build(ref=True)
    n, dx, org = (24, 20, 18), (10.0, 12.0, 13.0), (-120.0, -110.0, -100.0)
    np.testing.assert_array_equal(oracle.ic_random_seeds(n, dx, org, 0.3, 0.1),
                                  oracle.ref_random_seeds(n, dx, org, 0.3, 0.1, str(tmp_path)))
