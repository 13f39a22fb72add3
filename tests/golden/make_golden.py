"""Regenerate the golden fixtures in this directory (run in a container that has
the reference tree; the GPU box only reads the committed files).

  tungsten_norms_32.json  -- the regression norms of the reference's Tungsten test,
                             parsed from apps/tungsten/tests/test_tungsten.cpp
                             (values at :288-300, tolerance at :347,353).
  random_seeds.npz        -- the RandomSeeds initial condition on the two domains
                             of tests/unit/frontend/field_modifiers/
                             test_ic_random_seeds.cpp (32^3 spacing 8 and 16^3
                             spacing 16, origin -128), evaluated with the
                             reference's own Seed class (oracle/_ref/ref_seeds).
  tungsten_ops_16x12x10.npz -- filterMF / exp_Ldt / n_weight and the derived
                             parameters computed by the reference's own header-only
                             code (oracle/_ref/ref_ops, built by oracle/Makefile from
                             tungsten_spectral.hpp, tungsten_etd_workspace.hpp,
                             spectral_exp_coefficients.hpp, kspace.hpp).

usage: python tests/golden/make_golden.py [REFERENCE_TREE]
(default: $OPENPFC_REFERENCE_DIR, else the oracle build recipe's default mount)
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


RANDOM_SEEDS_CASES = {  # test_ic_random_seeds.cpp: "Field Application", "Integration with Model"
    "n32": ((32, 32, 32), (8.0, 8.0, 8.0), (-128.0, -128.0, -128.0), 0.5, 0.2),
    "n16": ((16, 16, 16), (16.0, 16.0, 16.0), (-128.0, -128.0, -128.0), 0.65, 0.15),
}


def random_seeds(ref_root):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={ref_root}"],
                   check=True)
    from oracle import oracle as O
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for key, (n, dx, org, rho, amp) in RANDOM_SEEDS_CASES.items():
            out[key] = O.ref_random_seeds(n, dx, org, rho, amp, td)
    np.savez_compressed(os.path.join(HERE, "random_seeds.npz"), **out)


if __name__ == "__main__":
    from oracle import oracle as O
    ref_root = sys.argv[1] if len(sys.argv) > 1 else O.reference_dir()
    if not ref_root:
        sys.exit("reference tree not found: pass it or set OPENPFC_REFERENCE_DIR")
    norms(ref_root)
    ops(ref_root)
    random_seeds(ref_root)
    print("golden fixtures written to", HERE)
