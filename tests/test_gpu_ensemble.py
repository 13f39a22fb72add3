"""Uneven-size ensemble (one persistent kernel per stage, n-step CUDA graph)
against the FP64 oracle, member by member.  Sides are drawn from
{32, 48, 64, 80, 96}; r ~ U(-0.35, -0.10), n0 ~ U(-0.35, -0.20), noise
U(-0.01, 0.01) -- the parameter-sweep configuration at a reduced member count."""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3


def members(count, seed, cubes=True):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        if cubes:
            s = int(rng.choice([32, 48, 64, 80, 96]))
            n = (s, s, s)
        else:
            n = (int(rng.choice([32, 48, 64, 80, 96])), int(rng.choice([16, 32, 48, 64, 80, 96, 128])),
                 int(rng.choice([32, 48, 64, 80, 96])))
        out.append({"n": n, "dx": PI4, "r": float(rng.uniform(-0.35, -0.10)),
                    "n0": float(rng.uniform(-0.35, -0.20)), "seed": 1000 + i})
    return out


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("cubes", [True, False])
def test_ensemble_vs_oracle(oracle, prec, tol, cubes):
    ms = members(12, 7 if cubes else 8, cubes)
    e = ob.Ensemble(ms, precision=prec)
    e.initialize(0.5)
    psi0 = [ob.ic_noise(m["n"], m["n0"], 0.01, m["seed"]) for m in ms]
    for i, p in enumerate(psi0):
        e.set_psi(i, p)
    e.step(10)
    e.sync()
    for i, m in enumerate(ms):
        ref = oracle.run_plain(psi0[i], PI4, m["r"], 0.5, 10)
        assert rel_l2(e.get_psi(i), ref) <= tol, (i, m["n"])


def test_ensemble_autotune_keeps_results(oracle, tmp_path, monkeypatch):
    monkeypatch.setenv("OPENPFC_GPU_AUTOTUNE_CACHE_DIR", str(tmp_path))
    ms = members(6, 9)
    e = ob.Ensemble(ms, precision=ob.FP32)
    e.initialize(0.5)
    mc, mx, mu = e.autotune()
    assert all(min(v for v in ms if v > 0) > 0 for ms in (mc, mx, mu))
    assert all(0 <= v < 6 for v in e.variants())
    psi0 = [ob.ic_noise(m["n"], m["n0"], 0.01, m["seed"]) for m in ms]
    for i, p in enumerate(psi0):
        e.set_psi(i, p)
    e.step(5)
    e.sync()
    for i, m in enumerate(ms):
        ref = oracle.run_plain(psi0[i], PI4, m["r"], 0.5, 5)
        assert rel_l2(e.get_psi(i), ref) <= 1e-5
