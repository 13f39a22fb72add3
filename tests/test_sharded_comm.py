"""The sharded decomposition's host side on CPU: the z-slab <-> kx-slab
transposes (with the extra column every block carries) against numpy, with P
ranks emulated in one process and with two gloo ranks exchanging their blocks
through the same TorchComm the GPU path uses (pairwise send/receive: gloo has no
all-to-all)."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _full_spectrum(n0, n1, n2, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n2, n1, n0 // 2 + 1, 2))


@pytest.mark.parametrize("P", [1, 2, 4])
def test_transposes_round_trip_local(P):
    import torch
    from openpfc_b200.sharded import LocalComm, kx_from_blocks, kx_to_z, z_from_blocks, z_to_kx
    n0, n1, n2 = 32, 8, 16
    M, Mloc, n2loc = n0 // 2, n0 // 2 // P, n2 // P
    whole = _full_spectrum(n0, n1, n2, 3)
    zfull = [torch.tensor(whole[q * n2loc:(q + 1) * n2loc]) for q in range(P)]
    comm = LocalComm(P)
    recvs = comm.alltoall([z_to_kx(z, P, Mloc) for z in zfull])
    kx = []
    for r in range(P):
        t = torch.zeros((n2, n1, Mloc + 1, 2), dtype=torch.float64)
        kx_from_blocks(recvs[r], t)
        # rank r holds global columns [r Mloc, r Mloc + Mloc], the last one being
        # the next rank's first column or, on the last rank, the Nyquist plane
        np.testing.assert_array_equal(t.numpy(), whole[:, :, r * Mloc:r * Mloc + Mloc + 1])
        kx.append(t)
    back = comm.alltoall([kx_to_z(t, P) for t in kx])
    for q in range(P):
        t = torch.zeros((n2loc, n1, M + 1, 2), dtype=torch.float64)
        z_from_blocks(back[q], t, Mloc)
        np.testing.assert_array_equal(t.numpy(), whole[q * n2loc:(q + 1) * n2loc])


SCRIPT = textwrap.dedent('''
    import sys, numpy as np, torch, torch.distributed as dist
    sys.path.insert(0, {root!r})
    from openpfc_b200.sharded import TorchComm, kx_from_blocks, kx_to_z, z_from_blocks, z_to_kx
    dist.init_process_group("gloo")
    comm = TorchComm()
    P, q = comm.size, comm.rank
    n0, n1, n2 = 32, 8, 16
    M, Mloc, n2loc = n0 // 2, n0 // 2 // P, n2 // P
    whole = np.random.default_rng(3).standard_normal((n2, n1, M + 1, 2))
    z = torch.tensor(whole[q * n2loc:(q + 1) * n2loc])
    (recv,) = comm.alltoall([z_to_kx(z, P, Mloc)])
    kx = torch.zeros((n2, n1, Mloc + 1, 2), dtype=torch.float64)
    kx_from_blocks(recv, kx)
    assert np.array_equal(kx.numpy(), whole[:, :, q * Mloc:q * Mloc + Mloc + 1])
    (back,) = comm.alltoall([kx_to_z(kx, P)])
    zz = torch.zeros_like(z)
    z_from_blocks(back, zz, Mloc)
    assert np.array_equal(zz.numpy(), z.numpy())
    total = comm.allreduce_sum([float(q + 1)])[0]
    assert total == P * (P + 1) / 2
    print("rank", q, "ok", flush=True)
    dist.destroy_process_group()
''')


def test_transposes_over_gloo_ranks(tmp_path):
    script = tmp_path / "a2a.py"
    script.write_text(SCRIPT.format(root=ROOT))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                        "--master-addr=127.0.0.1", "--master-port=29533", str(script)],
                       capture_output=True, text=True, timeout=180, env=env)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    assert p.stdout.count("ok") == 2
