"""Parity at the measured sizes: the plain conserved PFC step of
docs/api/examples/10_complete_pfc_model.cpp:121-144 at 256^3 and 512^3
(dx = pi/4, dt = 0.5, r = -0.25, psi0 = -0.285 + U(-0.01, 0.01), seed 7)
against the FP64 oracle, through the C ABI.

Each size runs with the kernel variants the autotuner picks on this GPU and
with variant sets forced through OPFC_{Y,X,Z}_VARIANT: the ping-pong y pass
(3), the register-loaded x pass (3) and the z update on the folded FP64-built
tables (6, 8: the FP32 candidates by default, 8 with the x pass prefetching the
next row, 4; 9: the 128-byte-row variant, which at these z lengths takes the
direct-load kernel) or on FP32-computed operators (5, an opt-in).  At these sizes every persistent CTA walks many tiles, and the y pass
has 512-point lines.  Tolerances: relative L2 over all cells <= 1e-11 (FP64),
<= 1e-5 (FP32).
"""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3
TOL = {ob.FP64: 1e-11, ob.FP32: 1e-5}

VARIANTS = {
    "autotuned": None,
    "y3x3z6": {"OPFC_Y_VARIANT": "3", "OPFC_X_VARIANT": "3", "OPFC_Z_VARIANT": "6"},
    "y3x3z5": {"OPFC_Y_VARIANT": "3", "OPFC_X_VARIANT": "3", "OPFC_Z_VARIANT": "5"},
    "y3x4z8": {"OPFC_Y_VARIANT": "3", "OPFC_X_VARIANT": "4", "OPFC_Z_VARIANT": "8"},
    "y3x4z9": {"OPFC_Y_VARIANT": "3", "OPFC_X_VARIANT": "4", "OPFC_Z_VARIANT": "9"},
}


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def cases(oracle):
    """Initial fields and oracle trajectories, computed once per module."""
    out = {}
    for n, steps in ((256, 20), (512, 3)):
        psi0 = oracle.ic_noise((n, n, n), -0.285, 0.01, 7)
        out[n] = (psi0, steps, oracle.run_plain(psi0, PI4, -0.25, 0.5, steps))
    return out


def _run(n, prec, psi0, steps, variant, monkeypatch, tmp_path):
    for k in ("OPFC_Y_VARIANT", "OPFC_X_VARIANT", "OPFC_Z_VARIANT", "OPFC_NO_TMA"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setenv("OPENPFC_GPU_AUTOTUNE_CACHE_DIR", str(tmp_path))
    monkeypatch.delenv("OPENPFC_GPU_AUTOTUNE_MODE", raising=False)
    env = VARIANTS[variant]
    if env:
        for k, v in env.items():
            monkeypatch.setenv(k, v)
    m = ob.PfcB200((n, n, n), PI4, r=-0.25, precision=prec)
    m.initialize(0.5)
    if env is None:
        m.autotune()
    else:
        yv, xv, zv = m.variants()
        assert (yv, xv, zv) == (int(env["OPFC_Y_VARIANT"]), int(env["OPFC_X_VARIANT"]), int(env["OPFC_Z_VARIANT"]))
    m.set_psi(psi0)
    m.step(steps)
    m.sync()
    return m


@pytest.mark.parametrize("variant", list(VARIANTS))
@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
@pytest.mark.parametrize("n", [256, 512])
def test_plain_config2_vs_oracle(cases, monkeypatch, tmp_path, n, prec, variant):
    psi0, steps, ref = cases[n]
    m = _run(n, prec, psi0, steps, variant, monkeypatch, tmp_path)
    err = rel_l2(m.get_psi(), ref)
    assert err <= TOL[prec], (n, prec, variant, m.variants(), err)
    # the k = 0 mode is carried in FP64: the mean density is the initial one
    assert abs(m.mass() - float(np.mean(psi0))) <= 1e-14


def test_fp32_vs_fp64_512_100_steps(cases, monkeypatch, tmp_path):
    """The measured configuration's accuracy claim: FP32 after 100 steps within
    1e-5 relative L2 of the FP64 GPU step (FP64 itself matches the oracle to
    1e-11 above), both with their autotuned variants."""
    psi0, _, _ = cases[512]
    m32 = _run(512, ob.FP32, psi0, 100, "autotuned", monkeypatch, tmp_path)
    a = m32.get_psi()
    del m32
    m64 = _run(512, ob.FP64, psi0, 100, "autotuned", monkeypatch, tmp_path)
    b = m64.get_psi()
    assert rel_l2(a, b) <= 1e-5
