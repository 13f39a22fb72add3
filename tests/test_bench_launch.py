"""The bench launcher on the CPU: `--gpus 2` starts two ranks by itself (gloo
dry run, no GPU work), and the reference arm runs the oracle's CPU step without
loading the product library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out):
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert lines, out
    return json.loads(lines[-1])


def test_gpus_2_starts_two_ranks():
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-run"],
                       capture_output=True, text=True, timeout=180, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = _last_json(p.stdout)
    assert line["n_gpus"] == 2
    assert line["config"]["parallelism"] == "replicas x2"


def test_reference_arm_does_not_load_the_product():
    code = ("import sys, bench; rc = bench.main(['--impl', 'reference', '--n', '16', '--steps', '2', "
            "'--warmup', '3']); assert rc == 0; "
            "assert not any(m == 'openpfc_b200' or m.startswith('openpfc_b200.') for m in sys.modules), "
            "sorted(m for m in sys.modules if 'openpfc' in m)")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=180, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    line = _last_json(p.stdout)
    assert line["impl"] == "reference" and line["n_gpus"] == 0
    assert line["warmup"] == 3 and line["steps"] == 2
