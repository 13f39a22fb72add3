"""On-disk formats of the reference's writers and readers, host side (no GPU):
file-name patterns (pfc::utils::format_with_number), raw binary boxes
(BinaryWriter / BinaryReader) and VTK ImageData (VTKWriter), through the C ABI
and the C++ mirrors."""
import os
import subprocess

import numpy as np
import pytest

import openpfc_b200 as ob
from openpfc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "openpfc_b200")


@pytest.mark.parametrize("pattern,inc,expect", [
    ("output_%d.dat", 0, "output_0.dat"), ("output_%d.dat", 12, "output_12.dat"),
    ("frame_%04d.vti", 7, "frame_0007.vti"), ("result_%-5d.bin", 1, "result_1    .bin"),
    ("r_%+d", 3, "r_+3"), ("plain.bin", 5, "plain.bin")])
def test_format_with_number(pattern, inc, expect):
    assert ob.format_with_number(pattern, inc) == expect


@pytest.mark.parametrize("pattern", ["a_%s.bin", "a_%d_%d.bin", "a_%n", "a_%f", "%", "a_%x.bin", "a_%%d"])
def test_format_with_number_rejects(pattern):
    with pytest.raises(ValueError):
        ob.format_with_number(pattern, 1)


def _i3(v):
    import ctypes
    return (ctypes.c_int * 3)(*v)


def test_raw_box_round_trip(tmp_path):
    L = _lib.lib()
    g = (6, 5, 4)
    a = np.arange(np.prod(g), dtype=np.float64).reshape(g[::-1]) * 0.5 - 7
    fn = str(tmp_path / "psi.bin").encode()
    assert L.opfc_write_raw(fn, _i3(g), _i3(g), _i3((0, 0, 0)), ob._dp(a), 1) == 0
    np.testing.assert_array_equal(np.fromfile(fn.decode(), dtype=np.float64).reshape(a.shape), a)
    # a box of the same file
    box = np.zeros((2, 3, 4))
    assert L.opfc_read_raw(fn, _i3(g), _i3((4, 3, 2)), _i3((1, 2, 1)), ob._dp(box), 1) == 0
    np.testing.assert_array_equal(box, a[1:3, 2:5, 1:5])
    # out-of-grid boxes and short files are refused
    assert L.opfc_read_raw(fn, _i3(g), _i3((4, 3, 2)), _i3((3, 2, 1)), ob._dp(box), 1) == -1
    big = np.zeros((5, 5, 6))
    assert L.opfc_read_raw(fn, _i3((6, 5, 5)), _i3((6, 5, 5)), _i3((0, 0, 0)), ob._dp(big), 1) == -2
    assert L.opfc_write_raw(str(tmp_path / "no" / "dir.bin").encode(), _i3(g), _i3(g), _i3((0, 0, 0)),
                            ob._dp(a), 1) == -8


def test_two_writers_fill_one_file(tmp_path):
    """Two writers, each with half of the global box (split along z and, in a
    second file, along x), fill one file whose contents equal the whole array;
    a stale longer file is truncated by the one-time prepare."""
    L = _lib.lib()
    g = (6, 5, 4)
    a = np.arange(np.prod(g), dtype=np.float64).reshape(g[::-1]) * 0.25 + 1
    for name, boxes in (("z", [((6, 5, 2), (0, 0, 0)), ((6, 5, 2), (0, 0, 2))]),
                        ("x", [((3, 5, 4), (3, 0, 0)), ((3, 5, 4), (0, 0, 0))])):
        fn = str(tmp_path / f"half_{name}.bin").encode()
        np.zeros(1000).tofile(fn.decode())  # stale, longer file under the same name
        assert L.opfc_prepare_raw(fn, _i3(g), 1) == 0
        for loc, off in boxes:  # later writers never truncate what earlier ones wrote
            part = np.ascontiguousarray(a[off[2]:off[2] + loc[2], off[1]:off[1] + loc[1],
                                          off[0]:off[0] + loc[0]])
            assert L.opfc_write_raw(fn, _i3(g), _i3(loc), _i3(off), ob._dp(part), 1) == 0
        got = np.fromfile(fn.decode(), dtype=np.float64)
        assert got.size == a.size
        np.testing.assert_array_equal(got.reshape(a.shape), a)


def test_cpp_io_mirrors(tmp_path):
    src = os.path.join(ROOT, "tests", "cpp", "test_io.cpp")
    exe = str(tmp_path / "test_io")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), src,
                    "-L", LIBDIR, "-lopenpfc_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
