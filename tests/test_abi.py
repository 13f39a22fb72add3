"""CPU checks of the C-ABI library: it loads, exports every symbol the public
header declares, and its host-only entry points behave (no GPU compute here)."""
import ctypes
import os
import subprocess

import pytest

import openpfc_b200 as ob
import numpy as np
from openpfc_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_exported_symbols_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for s in _lib.declared_symbols():
        assert s in names, s


def test_status_strings_and_defaults():
    L = _lib.lib()
    assert L.opfc_status_string(0) == b"ok"
    assert L.opfc_status_string(-2) == b"size contract violated"
    d = ob.default_desc()
    # TungstenParams defaults, tungsten_params.hpp:33-57
    assert d.tungsten.n0 == -0.10 and d.tungsten.T == 3300.0 and d.tungsten.alpha_highOrd == 4
    assert d.tungsten.lambda_ == 0.22 and d.tungsten.q40 == 45.0
    assert d.precision == ob.FP32 and d.r == -0.25


def test_bad_descriptor_rejected_before_device_use():
    L = _lib.lib()
    h = ctypes.c_void_p()
    d = ob.default_desc()
    d.n[0] = 7  # odd x extent: no R2C layout
    assert L.opfc_create(ctypes.byref(d), ctypes.byref(h)) == -2
    d = ob.default_desc()
    d.n[1] = 100  # unsupported transform length
    assert L.opfc_create(ctypes.byref(d), ctypes.byref(h)) == -2
    d = ob.default_desc()
    d.precision = 7
    assert L.opfc_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert L.opfc_create(None, ctypes.byref(h)) == -1


def test_header_has_no_forbidden_copy_calls():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, "openpfc_b200", "csrc", "opfc.cu")).read()
    assert "Batch" + "Async" not in src


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="host without a GPU only")
def test_create_without_gpu_reports_cuda_error():
    h = ctypes.c_void_p()
    d = ob.default_desc()
    d.n[0] = d.n[1] = d.n[2] = 8
    rc = _lib.lib().opfc_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == -3 and not h.value


def test_ic_generators_match_oracle(oracle):
    import math
    import numpy as np
    n = (12, 10, 8)
    np.testing.assert_array_equal(ob.ic_noise(n, -0.285, 0.01, 42), oracle.ic_noise(n, -0.285, 0.01, 42))
    dx = [math.pi / 4] * 3
    np.testing.assert_array_equal(ob.ic_seeds(n, dx, -0.1, 0.001, 3, 3.0, 0.2, 9),
                                  oracle.ic_seeds(n, dx, -0.1, 0.001, 3, 3.0, 0.2, 9))
    # seeds straddling the periodic boundary, radius well below the box
    for seed in (1, 2, 3):
        m = (48, 40, 32)
        np.testing.assert_array_equal(ob.ic_seeds(m, dx, -0.1, 0.001, 6, 7.5, 0.2, seed),
                                      oracle.ic_seeds(m, dx, -0.1, 0.001, 6, 7.5, 0.2, seed))
    d = 1.1107207345395915
    origin = [-0.5 * d * 16] * 3
    a = ob.ic_seed(np.full((16, 16, 16), -0.4), [d] * 3, origin, [0, 0, 0], 8.0, -0.047, 0.215936)
    b = oracle.ic_seed_inside(np.full((16, 16, 16), -0.4), [d] * 3, origin, 8.0, -0.047, 0.215936)
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-15)


def test_seed_grid_fcc_matches_oracle(oracle):
    # the Aluminum test's initial condition (apps/aluminumNew/aluminumTest.cpp:83-96)
    import numpy as np
    base = np.full((32, 32, 32), -0.0060)
    a = ob.ic_seed_grid_fcc(base, [1.0] * 3, [0.0] * 3, 1, 2, 2, 8.0, 4.0, 0.4, -0.036, 42)
    b = oracle.ic_seed_grid_fcc(base, [1.0] * 3, [0.0] * 3, 1, 2, 2, 8.0, 4.0, 0.4, -0.036, 42)
    np.testing.assert_array_equal(a, b)
    assert abs(float((a ** 2).sum()) - 1297.08) <= 0.1
    # anisotropic spacing, offset origin, several seeds
    base = np.full((20, 24, 28), 0.1)
    a = ob.ic_seed_grid_fcc(base, [0.7, 0.9, 1.1], [-2.0, 1.0, 0.5], 1, 3, 2, 6.0, 5.0, 0.3, -0.05, 7)
    b = oracle.ic_seed_grid_fcc(base, [0.7, 0.9, 1.1], [-2.0, 1.0, 0.5], 1, 3, 2, 6.0, 5.0, 0.3, -0.05, 7)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("key,case", [
    ("n32", ((32, 32, 32), (8.0, 8.0, 8.0), (-128.0, -128.0, -128.0), 0.5, 0.2)),
    ("n16", ((16, 16, 16), (16.0, 16.0, 16.0), (-128.0, -128.0, -128.0), 0.65, 0.15))])
def test_random_seeds_matches_reference_fixture(oracle, golden_dir, key, case):
    """The product's RandomSeeds equals the reference-Seed fixture and the
    oracle bit for bit (the domains of test_ic_random_seeds.cpp)."""
    n, dx, org, rho, amp = case
    got = ob.ic_random_seeds(n, dx, org, rho, amp)
    np.testing.assert_array_equal(got, np.load(os.path.join(golden_dir, "random_seeds.npz"))[key])
    np.testing.assert_array_equal(got, oracle.ic_random_seeds(n, dx, org, rho, amp))


def test_step_kernel_regions_name_the_reference_regions():
    L = _lib.lib()
    names = [L.opfc_step_kernel_name(k).decode() for k in range(5)]
    regions = [L.opfc_step_kernel_region(k).decode() for k in range(5)]
    assert names == ["y_inverse", "x_fused", "y_forward", "z_update", "hermitian_fix"]
    # every kernel sits in a region of the reference's step (tungsten_model.hpp:313-362)
    assert all(r.startswith("gradient/mean_field/") or r.startswith("gradient/evolve/") for r in regions)
    assert "gradient/evolve/forward + multiply + backward" in regions[3]
    assert L.opfc_step_kernel_region(5) == b"" and L.opfc_step_kernel_region(-1) == b""
