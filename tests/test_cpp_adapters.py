"""The C++ drop-in adapters (include/openpfc_b200/pfc_b200.hpp): they compile
and link against the C-ABI library on any host; on a GPU the test program runs
the reference's FFT known answers and Tungsten golden norms through them."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_adapters.cpp")
LIBDIR = os.path.join(ROOT, "openpfc_b200")


def build(tmpdir):
    exe = os.path.join(tmpdir, "test_adapters")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lopenpfc_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe],
                   check=True, capture_output=True, text=True)
    return exe


def test_adapters_compile_and_link(tmp_path):
    assert os.path.exists(build(str(tmp_path)))


@pytest.mark.gpu
def test_adapters_run_reference_checks(tmp_path):
    exe = build(str(tmp_path))
    r = subprocess.run([exe, os.path.join(ROOT, "tests", "golden", "tungsten_norms_32.json")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
