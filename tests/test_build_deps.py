"""The in-place build recompiles an object when a header it was built from
changes: the headers come from nvcc's -MD file next to the object, and every
project header is assumed when that file is missing or names a header that no
longer exists."""
import os

from openpfc_b200 import build


def test_deps_from_dependency_file(tmp_path, monkeypatch):
    monkeypatch.setattr(build, "ROOT", str(tmp_path))
    src = tmp_path / "a.cu"
    hdr = tmp_path / "b.cuh"
    src.write_text("")
    hdr.write_text("")
    obj = tmp_path / "a.o"
    (tmp_path / "a.d").write_text(f"{obj}: {src} \\\n {hdr} \\\n /usr/include/stdio.h\n")
    assert build._deps(str(obj), "a.cu") == [str(src), str(hdr)]


def test_deps_fall_back_to_every_header(tmp_path):
    obj = tmp_path / "kernels_f32.o"
    deps = build._deps(str(obj), "kernels_f32.cu")  # no .d file
    assert os.path.join(build.CSRC, "kernels_f32.cu") in deps
    assert all(os.path.join(build.CSRC, h) in deps for h in build.HEADERS)
    (tmp_path / "kernels_f32.d").write_text(f"{obj}: {tmp_path}/gone.cuh\n")
    assert os.path.join(build.CSRC, "kernels.cuh") in build._deps(str(obj), "kernels_f32.cu")


def test_stale(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    a.write_text("")
    b.write_text("")
    os.utime(a, (1000, 1000))
    os.utime(b, (2000, 2000))
    assert build._stale(str(a), [str(b)])
    assert not build._stale(str(b), [str(a)])
    assert build._stale(str(tmp_path / "missing.o"), [str(a)])
