"""Regenerate the golden fixtures in this directory (run in a container that has
the reference tree; the GPU box only reads the committed files).

  tungsten_norms_32.json  -- the regression norms of the reference's Tungsten test,
                             parsed from apps/tungsten/tests/test_tungsten.cpp
                             (values at :288-300, tolerance at :347,353).
  tungsten_ops_16x12x10.npz -- filterMF / exp_Ldt / n_weight and the derived
                             parameters computed by the reference's own header-only
                             code (oracle/_ref/ref_ops, built by oracle/Makefile from
                             tungsten_spectral.hpp, tungsten_etd_workspace.hpp,
                             spectral_exp_coefficients.hpp, kspace.hpp).

usage: python tests/golden/make_golden.py [/root/reference]
"""
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def norms(ref_root):
    path = os.path.join(ref_root, "apps/tungsten/tests/test_tungsten.cpp")
    txt = open(path).read()
    block = re.search(r"expected_norms\{(.*?)\};", txt, re.S).group(1)
    vals = [float(v) for v in re.findall(r"([0-9]+\.[0-9]+)", block)]
    assert len(vals) == 11, vals
    out = {
        "source": "apps/tungsten/tests/test_tungsten.cpp:288-300 (tolerance :347,353)",
        "grid": [32, 32, 32], "dx": 1.1107207345395915, "dt": 1.0,
        "ic": {"constant": -0.4, "seed_radius": 18.0, "rho_seed": -0.047, "amp_eq": 0.215936,
               "origin": "-0.5*dx*32 per axis"},
        "abs_tol": 0.1,
        "norms": vals,
    }
    with open(os.path.join(HERE, "tungsten_norms_32.json"), "w") as f:
        json.dump(out, f, indent=1)


def ops(ref_root):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={ref_root}"],
                   check=True)
    from oracle import oracle as O
    n, dx, dt = (16, 12, 10), 1.1107207345395915, 1.0
    with tempfile.TemporaryDirectory() as td:
        r = O.ref_ops(n, dx, dt, td)
    np.savez_compressed(os.path.join(HERE, "tungsten_ops_16x12x10.npz"), n=np.array(n), dx=dx, dt=dt,
                        derived=r["derived"], filterMF=r["filterMF"], exp_Ldt=r["exp_Ldt"],
                        n_weight=r["n_weight"])


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    norms(ref_root)
    ops(ref_root)
    print("golden fixtures written to", HERE)
