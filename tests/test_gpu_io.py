"""Handle-level files: the field written by opfc_write_binary / opfc_write_vti
is the field opfc_get_psi returns (bit for bit, FP64), and opfc_read_binary
restores a state whose first step matches the oracle."""
import math

import numpy as np
import pytest

import openpfc_b200 as ob

pytestmark = pytest.mark.gpu
PI4 = [math.pi / 4] * 3


@pytest.mark.parametrize("prec", [ob.FP64, ob.FP32])
def test_binary_and_vti_round_trip(oracle, tmp_path, prec):
    n = (32, 24, 16)
    psi0 = oracle.ic_noise(n, -0.285, 0.01, 5)
    m = ob.PfcB200(n, PI4, precision=prec, origin=[-1.0, 0.5, 2.0])
    m.initialize(0.5)
    m.set_psi(psi0)
    m.step(3)
    m.sync()
    psi = m.get_psi()
    m.write_binary(str(tmp_path / "psi_%03d.bin"), 3)
    raw = np.fromfile(str(tmp_path / "psi_003.bin"), dtype=np.float64)
    np.testing.assert_array_equal(raw.reshape(psi.shape), psi)
    m.write_binary_hat(str(tmp_path / "hat.bin"))
    hat = np.fromfile(str(tmp_path / "hat.bin"), dtype=np.complex128)
    np.testing.assert_array_equal(hat.reshape(n[2], n[1], n[0] // 2 + 1), m.get_psi_hat())
    m.write_vti(str(tmp_path / "f_%d.vti"), 1, "psi")
    vti = open(tmp_path / "f_1.vti", "rb").read()
    head, rest = vti.split(b"<AppendedData encoding=\"raw\">\n_", 1)
    assert b'WholeExtent="0 31 0 23 0 15" Origin="-1 0.5 2" Spacing="0.785398 0.785398 0.785398"' in head
    assert int(np.frombuffer(rest[:8], dtype=np.uint64)[0]) == psi.size * 8
    np.testing.assert_array_equal(np.frombuffer(rest[8:8 + psi.size * 8], dtype=np.float64).reshape(psi.shape), psi)
    # FileReader: restart from the file, one step, against the oracle
    m2 = ob.PfcB200(n, PI4, precision=prec)
    m2.initialize(0.5)
    m2.read_binary(str(tmp_path / "psi_003.bin"))
    if prec == ob.FP64:  # the state goes through a forward and an inverse transform
        np.testing.assert_allclose(m2.get_psi(), psi, rtol=0, atol=1e-14)
    m2.step(1)
    m2.sync()
    ref = oracle.run_plain(psi, PI4, -0.25, 0.5, 1)
    tol = 1e-12 if prec == ob.FP64 else 1e-5
    assert np.linalg.norm((m2.get_psi() - ref).ravel()) <= tol * np.linalg.norm(ref.ravel())


def test_read_binary_short_file(tmp_path):
    n = (16, 16, 16)
    m = ob.PfcB200(n, PI4, precision=ob.FP64)
    m.initialize(0.5)
    np.zeros(100).tofile(str(tmp_path / "short.bin"))
    with pytest.raises(ValueError):  # OPFC_ERR_SIZE, like std::invalid_argument
        m.read_binary(str(tmp_path / "short.bin"))
    with pytest.raises(ob.OpfcError):
        m.write_binary(str(tmp_path / "bad_%s.bin"))
