"""Both kernel families against the oracle: the persistent TMA/bulk-copy-fed
passes (default) and the direct-load passes (OPFC_NO_TMA=1, read at handle
creation), for every model and both precisions."""
import math
import os

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu

PI4 = [math.pi / 4] * 3


@pytest.fixture(params=["tma", "tma_radial", "direct", "computed", "direct_computed", "pingpong", "e32",
                        "folded", "folded_direct", "folded_nopp", "folded_wide"])
def path(request, monkeypatch):
    """tma: pipelined kernels streaming the per-mode tables (default);
    tma_radial: the z update reading radial operator tables (OPFC_Z_VARIANT=1,
    isotropic grids; others fall back to tables);
    direct: direct-load kernels (OPFC_NO_TMA=1);
    computed: pipelined z update computing its operators from k^2
    (OPFC_Z_VARIANT=3), half-width y tiles (OPFC_Y_VARIANT=2) and the x pass
    without the warp-square kernel (OPFC_X_VARIANT=2);
    direct_computed: direct z update computing its operators (OPFC_Z_VARIANT=4);
    pingpong: ping-pong FFT exchange buffers in the y pass and the computed
    z update (OPFC_Y_VARIANT=3, OPFC_Z_VARIANT=5), and the x pass's warp-square
    kernel with rows loaded straight into registers (OPFC_X_VARIANT=3);
    e32: direct-load y pass with 32 values per thread (OPFC_Y_VARIANT=4;
    other lengths keep their plan);
    folded: the z update reading the folded FP64-built tables with ping-pong
    exchange buffers, with the ping-pong y pass and the register-loaded x pass
    (OPFC_Y_VARIANT=3, OPFC_X_VARIANT=3, OPFC_Z_VARIANT=6);
    folded_direct: direct-load z update on the folded tables (OPFC_Z_VARIANT=7);
    folded_nopp: pipelined z update on the folded tables without ping-pong
    buffers (OPFC_Z_VARIANT=8) with the register-loaded x pass prefetching the
    next row (OPFC_X_VARIANT=4);
    folded_wide: the z update on the folded tables with 128-byte tile rows
    streamed through a two-slot box ring (OPFC_Z_VARIANT=9; z lengths other
    than 1024 and the Tungsten model take the direct-load kernel).
    The Tungsten model has no computed operators and falls back to tables."""
    monkeypatch.delenv("OPFC_NO_TMA", raising=False)
    monkeypatch.delenv("OPFC_Z_VARIANT", raising=False)
    monkeypatch.delenv("OPFC_Y_VARIANT", raising=False)
    monkeypatch.delenv("OPFC_X_VARIANT", raising=False)
    monkeypatch.setenv("OPENPFC_GPU_AUTOTUNE_MODE", "fallback_only")
    if request.param == "direct":
        monkeypatch.setenv("OPFC_NO_TMA", "1")
    elif request.param == "tma_radial":
        monkeypatch.setenv("OPFC_Z_VARIANT", "1")
    elif request.param == "computed":
        monkeypatch.setenv("OPFC_Z_VARIANT", "3")
        monkeypatch.setenv("OPFC_Y_VARIANT", "2")
        monkeypatch.setenv("OPFC_X_VARIANT", "2")
    elif request.param == "direct_computed":
        monkeypatch.setenv("OPFC_Z_VARIANT", "4")
    elif request.param == "pingpong":
        monkeypatch.setenv("OPFC_Y_VARIANT", "3")
        monkeypatch.setenv("OPFC_Z_VARIANT", "5")
        monkeypatch.setenv("OPFC_X_VARIANT", "3")
    elif request.param == "e32":
        monkeypatch.setenv("OPFC_Y_VARIANT", "4")
    elif request.param == "folded":
        monkeypatch.setenv("OPFC_Y_VARIANT", "3")
        monkeypatch.setenv("OPFC_X_VARIANT", "3")
        monkeypatch.setenv("OPFC_Z_VARIANT", "6")
    elif request.param == "folded_direct":
        monkeypatch.setenv("OPFC_Z_VARIANT", "7")
    elif request.param == "folded_nopp":
        monkeypatch.setenv("OPFC_Z_VARIANT", "8")
        monkeypatch.setenv("OPFC_X_VARIANT", "4")
    elif request.param == "folded_wide":
        monkeypatch.setenv("OPFC_Z_VARIANT", "9")
    return request.param


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("n", [(64, 64, 64), (128, 32, 256), (256, 16, 512), (512, 32, 16), (1024, 16, 16),
                               (16, 512, 512), (32, 128, 128), (32, 16, 1024), (32, 1024, 16)])
def test_plain(oracle, path, prec, tol, n):
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 3)
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 10)
    m = ob.PfcB200(n, PI4, precision=prec)
    m.initialize(0.5)
    m.set_psi(psi0)
    m.step(10)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= tol


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("n", [(64, 64, 32), (512, 16, 16), (128, 32, 32), (1024, 16, 8), (16, 32, 1024)])
def test_filtered(oracle, path, prec, tol, n):
    psi0 = oracle.ic_seeds(n, PI4, -0.10, 0.001, 2, 8.0, 0.2, 4)
    ref = oracle.run_filtered(psi0, PI4, -0.3, 0.5, -0.1, -0.5, 0.3, 0.5, 10)
    m = ob.FilteredB200(n, PI4, precision=prec)
    m.initialize(0.5)
    m.set_psi(psi0)
    m.step(10)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= tol


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("n", [(64, 64, 64), (128, 64, 32), (512, 16, 32), (32, 16, 1024)])
def test_tungsten(oracle, path, prec, tol, n):
    dx = 1.1107207345395915
    psi0 = np.full((n[2], n[1], n[0]), -0.4)
    origin = [-0.5 * dx * n[a] for a in range(3)]
    psi0 = oracle.ic_seed_inside(psi0, [dx] * 3, origin, 20.0, -0.047, 0.215936)
    p = oracle.TungstenParams.defaults()
    ref = oracle.run_tungsten(psi0, [dx] * 3, p, 1.0, 5)
    m = ob.TungstenB200(n, [dx] * 3, precision=prec)
    m.initialize(1.0)
    m.set_psi(psi0)
    m.step(5)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= tol


def test_autotune_then_parity(oracle, tmp_path, monkeypatch):
    """The autotuner times every variant, picks one, and the tuned step still
    matches the oracle; a second handle reads the cached choice."""
    monkeypatch.setenv("OPENPFC_GPU_AUTOTUNE_CACHE_DIR", str(tmp_path))
    monkeypatch.delenv("OPENPFC_GPU_AUTOTUNE_MODE", raising=False)
    monkeypatch.delenv("OPFC_Z_VARIANT", raising=False)
    monkeypatch.delenv("OPFC_FP32_COMPUTED_OPERATORS", raising=False)
    n = (64, 64, 64)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 21)
    ref = oracle.run_plain(psi0, PI4, -0.25, 0.5, 10)
    m = ob.PfcB200(n, PI4, precision=ob.FP32)
    m.initialize(0.5)
    ms = m.autotune()
    assert ms["y.pipelined"] > 0 and ms["y.narrow"] > 0 and ms["z.tables"] > 0 and ms["z.radial"] > 0
    assert ms["z.folded_pingpong"] > 0 and ms["z.direct_folded"] > 0 and ms["z.folded"] > 0
    # FP32 operators computed per mode are candidates only on request
    assert ms["z.computed"] == -1 and ms["z.direct_computed"] == -1 and ms["z.computed_pingpong"] == -1
    assert m.variants()[2] not in (3, 4, 5)
    chosen = m.variants()
    m.set_psi(psi0)
    m.step(10)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= 1e-5
    assert any(f.name.endswith("_opfc_autotune.json") for f in tmp_path.iterdir())
    m2 = ob.PfcB200(n, PI4, precision=ob.FP32)
    m2.initialize(0.5)
    assert m2.variants() == chosen


def test_transforms(oracle, path):
    n = (128, 64, 512)
    x = np.random.default_rng(2).standard_normal((n[2], n[1], n[0]))
    f = ob.B200Fft(n, precision=ob.FP64)
    X = f.forward(x)
    Xo = oracle.r2c(x)
    assert np.abs(X - Xo).max() <= 1e-12 * np.abs(Xo).max()
    assert np.abs(f.backward(Xo) - oracle.c2r(Xo, n[0])).max() <= 1e-12 * np.abs(x).max()


def test_autotune_fp32_computed_operators_on_request(tmp_path, monkeypatch):
    monkeypatch.setenv("OPENPFC_GPU_AUTOTUNE_CACHE_DIR", str(tmp_path))
    monkeypatch.delenv("OPENPFC_GPU_AUTOTUNE_MODE", raising=False)
    monkeypatch.delenv("OPFC_Z_VARIANT", raising=False)
    monkeypatch.setenv("OPFC_FP32_COMPUTED_OPERATORS", "1")
    m = ob.PfcB200((64, 64, 64), PI4, precision=ob.FP32)
    m.initialize(0.5)
    ms = m.autotune()
    assert ms["z.computed"] > 0 and ms["z.direct_computed"] > 0 and ms["z.computed_pingpong"] > 0


@pytest.mark.parametrize("prec,tol", [(ob.FP64, 1e-11), (ob.FP32, 1e-5)])
@pytest.mark.parametrize("n", [(1024, 32, 32), (32, 1024, 32), (32, 32, 1024)])
def test_filtered_1024_axes(oracle, path, prec, tol, n):
    """Every axis at the measured filtered configuration's length (1024) once,
    with the others short: 1024-point x rows (M = 512), y lines and z lines
    (the z update's W = 4 tiles, its one- and two-stage rings, the (ky, N1 - ky)
    tile order over 1024 rows)."""
    psi0 = oracle.ic_seeds(n, PI4, -0.10, 0.001, 2, 8.0, 0.2, 6)
    ref = oracle.run_filtered(psi0, PI4, -0.3, 0.5, -0.1, -0.5, 0.3, 0.5, 6)
    m = ob.FilteredB200(n, PI4, precision=prec)
    m.initialize(0.5)
    m.set_psi(psi0)
    m.step(6)
    m.sync()
    assert rel_l2(m.get_psi(), ref) <= tol
