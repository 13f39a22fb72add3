"""Parity of the mean-field-filtered model with 1024-point z lines, the z length
of the filtered 1024^3 configuration, against the FP64 oracle through the C ABI.

Set-up:
- psi0 = -0.10 + U(-0.001, 0.001), then 8 seeds of radius 20 cells and
  amplitude 0.2 (seed 11);
- r = -0.3, alpha = 0.5, p2 = -0.1, p3 = -0.5, p4 = 0.3;
- dx = pi/4, dt = 0.5, 10 steps.

128 x 128 x 1024 keeps the oracle at a few seconds, while every CTA of the z
update walks many 1024-row tiles.

Each precision runs with the autotuner's pick and with the z update forced to
each of these, all on the folded FP64-built tables:
- the box-ring kernel with 128-byte tile rows (9);
- the ring-pipelined kernel (8);
- the direct-load kernel (7).

Tolerances: relative L2 over all cells <= 1e-11 (FP64), <= 1e-5 (FP32).
"""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3
SHAPE = (128, 128, 1024)
TOL = {ob.FP64: 1e-11, ob.FP32: 1e-5}
PARAMS = dict(r=-0.3, alpha=0.5, p2=-0.1, p3=-0.5, p4=0.3)


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="module")
def case(oracle):
    psi0 = oracle.ic_seeds(SHAPE, PI4, -0.10, 0.001, 8, 20.0, 0.2, 11)
    p = PARAMS
    ref = oracle.run_filtered(psi0, PI4, p["r"], p["alpha"], p["p2"], p["p3"], p["p4"], 0.5, 10)
    return psi0, ref


@pytest.mark.parametrize("z", [None, 9, 8, 7])
@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_filtered_1024_z_vs_oracle(case, monkeypatch, tmp_path, prec, z):
    psi0, ref = case
    for k in ("OPFC_Y_VARIANT", "OPFC_X_VARIANT", "OPFC_Z_VARIANT", "OPFC_NO_TMA"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setenv("OPENPFC_GPU_AUTOTUNE_CACHE_DIR", str(tmp_path))
    monkeypatch.delenv("OPENPFC_GPU_AUTOTUNE_MODE", raising=False)
    if z is not None:
        monkeypatch.setenv("OPFC_Z_VARIANT", str(z))
    m = ob.FilteredB200(SHAPE, PI4, precision=prec, **PARAMS)
    m.initialize(0.5)
    if z is None:
        ms = m.autotune()
        assert ms["z.folded_wide"] > 0
    else:
        assert m.variants()[2] == z
    m.set_psi(psi0)
    m.step(10)
    m.sync()
    err = rel_l2(m.get_psi(), ref)
    assert err <= TOL[prec], (prec, z, m.variants(), err)
