"""One field sharded over ranks: the sharded 3D FFT and PFC step.

The reference splits a field over MPI ranks and lets HeFFTe reshape it between
the decompositions each FFT direction needs (src/openpfc/runtime/cpu/fft.cpp:72-81,
its plan_options).  Here a grid N0 x N1 x N2 on P ranks is held

  * in z slabs for the x and y passes: rank q owns the planes
    z in [q N2/P, (q+1) N2/P) of the real field, and of the half spectrum
    transformed along x and y;
  * in kx slabs for the z transform and the z update: rank r owns the
    half-spectrum columns kx in [r M/P, (r+1) M/P), M = N0/2, for every ky and
    kz, and the last rank also the kx = M (Nyquist) plane,

with an all-to-all transpose between the two (two per PFC step, as the
reference's reshapes).  Each rank's compute runs in the library's kernels on two
handles -- a z-slab handle and a kx-slab handle whose operators use the global
wave numbers -- through opfc_pass; the transposes are tensor copies plus one
collective all-to-all: NCCL's on GPUs, pairwise send/receive on gloo, or plain
copies between the buffers of P ranks emulated in one process (LocalComm: the
1-GPU test of the whole decomposition).  Each block a rank sends holds M/P + 1
columns, the last one being the next rank's first column (or the Nyquist plane
for the last rank), so every pair exchanges the same number of bytes; a kx-slab
handle's own Nyquist plane thus holds a copy of the next rank's first column,
which it evolves like that rank and never sends back.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import FP32, FP64, MODEL_FILTERED, MODEL_PLAIN, _check, default_desc, lib

PASS_Y_INVERSE, PASS_X_FUSED, PASS_Y_FORWARD, PASS_Z_UPDATE = 0, 1, 2, 3
PASS_XY_FORWARD, PASS_XY_BACKWARD, PASS_Z_FORWARD, PASS_Z_INVERSE, PASS_Z_INVERSE_STATE = 4, 5, 6, 7, 8
ARRAY_WORK, ARRAY_STATE, ARRAY_REAL = 0, 1, 2

_SUPPORTED = (1, 2, 4, 8, 16, 24, 32, 40, 48, 64, 80, 96, 128, 256, 512, 1024)


class LocalComm:
    """P ranks emulated in one process: all of them are local, an all-to-all is
    a set of copies between their buffers."""

    def __init__(self, size: int):
        self.size = size
        self.local_ranks = list(range(size))

    def alltoall(self, sends):
        """sends[i][d]: block local rank i sends to rank d -> recvs[i][s]."""
        return [[sends[s][d] for s in range(self.size)] for d in range(self.size)]

    def allreduce_sum(self, values):
        return [math.fsum(values)] * self.size


class TorchComm:
    """One rank per process over torch.distributed: all_to_all on NCCL,
    pairwise isend / irecv on gloo (which has no all-to-all)."""

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist
        self.size = dist.get_world_size()
        self.rank = dist.get_rank()
        self.local_ranks = [self.rank]
        self.nccl = dist.get_backend() == "nccl"

    def alltoall(self, sends):
        import torch
        (send,) = sends
        recv = [torch.empty_like(send[s]) for s in range(self.size)]
        if self.nccl:
            self.dist.all_to_all(recv, [t.contiguous() for t in send])
        else:
            reqs = []
            for d in range(self.size):
                if d == self.rank:
                    recv[d].copy_(send[d])
                    continue
                reqs.append(self.dist.isend(send[d].contiguous(), d))
                reqs.append(self.dist.irecv(recv[d], d))
            for q in reqs:
                q.wait()
        return [recv]

    def allreduce_sum(self, values):
        import torch
        (v,) = values
        t = torch.tensor([v], dtype=torch.float64, device="cuda" if self.nccl else "cpu")
        self.dist.all_reduce(t)
        return [float(t.item())]


class _CudaArray:
    """A raw device pointer seen as a torch tensor (no copy)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None}


def z_to_kx(full_z, P, Mloc):
    """Blocks a z-slab rank sends: full_z is its half spectrum as (N2/P, N1, M+1, 2)
    (kx = M last); block r holds columns [r Mloc, r Mloc + Mloc] (Mloc + 1)."""
    return [full_z[:, :, r * Mloc:r * Mloc + Mloc + 1].contiguous() for r in range(P)]


def kx_from_blocks(recv, kx_full):
    """Assemble a kx-slab rank's (N2, N1, Mloc + 1, 2) columns from the blocks of
    every z-slab rank (stacked along z)."""
    n2loc = recv[0].shape[0]
    for q, b in enumerate(recv):
        kx_full[q * n2loc:(q + 1) * n2loc] = b


def kx_to_z(kx_full, P):
    """Blocks a kx-slab rank sends: its columns restricted to each z slab."""
    n2loc = kx_full.shape[0] // P
    return [kx_full[q * n2loc:(q + 1) * n2loc].contiguous() for q in range(P)]


def z_from_blocks(recv, full_z, Mloc):
    """Assemble a z-slab rank's (N2/P, N1, M+1, 2) half spectrum: the first Mloc
    columns of block r at [r Mloc, r Mloc + Mloc); the last rank's extra column
    is the Nyquist plane."""
    P = len(recv)
    for r, b in enumerate(recv):
        full_z[:, :, r * Mloc:(r + 1) * Mloc] = b[:, :, :Mloc]
    full_z[:, :, P * Mloc] = recv[P - 1][:, :, Mloc]


class _Rank:
    def __init__(self, owner, rank):
        self.rank = rank
        o = owner
        self.zs = _handle(o, (o.n[0], o.n[1], o.n2loc), 0)
        self.kx = _handle(o, (2 * o.mloc, o.n[1], o.n[2]), rank * o.mloc)

    def close(self):
        for h in (self.zs, self.kx):
            if h.value:
                lib().opfc_destroy(h)
                h.value = None


def _handle(o, n, kx0):
    d = default_desc()
    d.n[0], d.n[1], d.n[2] = n
    for a in range(3):
        d.dx[a] = float(o.dx[a])
        d.n_global[a] = int(o.n[a])
    d.kx0 = int(kx0)
    d.precision = o.precision
    d.model = o.model
    d.r = float(o.r)
    d.filter_alpha, d.p2, d.p3, d.p4 = float(o.alpha), float(o.p2), float(o.p3), float(o.p4)
    d.device = o.device
    d.stream = o.stream_handle
    h = ctypes.c_void_p()
    _check(None, lib().opfc_create(ctypes.byref(d), ctypes.byref(h)))
    return h


class ShardedPfc:
    """A plain (or filtered) PFC field on the ranks of `comm`, z slabs of the real
    field per rank.  N2 and N0/2 must divide by the number of ranks, and N2/P,
    N0/(2P) must be supported transform lengths.  All handles run on one CUDA
    stream per process, with the transposes' copies on the same stream."""

    def __init__(self, n, dx, comm, r=-0.25, precision=FP32, model="plain", alpha=0.5, p2=-0.1, p3=-0.5, p4=0.3,
                 device=0):
        import torch
        self.n = tuple(int(v) for v in n)
        self.dx = list(dx)
        self.comm = comm
        self.P = comm.size
        self.precision = precision
        self.model = MODEL_PLAIN if model == "plain" else MODEL_FILTERED
        self.r, self.alpha, self.p2, self.p3, self.p4 = r, alpha, p2, p3, p4
        self.device = device
        M = self.n[0] // 2
        if self.n[2] % self.P or M % self.P:
            raise ValueError("N2 and N0/2 must be multiples of the number of ranks")
        self.n2loc, self.mloc = self.n[2] // self.P, M // self.P
        if self.n2loc not in _SUPPORTED or self.mloc not in _SUPPORTED:
            raise ValueError("N2/P and N0/(2P) must be supported transform lengths")
        torch.cuda.set_device(device)
        self.stream = torch.cuda.Stream(device=device)
        self.stream_handle = ctypes.c_void_p(self.stream.cuda_stream)
        self.ranks = [_Rank(self, rk) for rk in comm.local_ranks]
        self.mean = 0.0
        self.dtype = torch.float64 if precision == FP64 else torch.float32
        self._typestr = "<f8" if precision == FP64 else "<f4"
        self._a_ready = False

    def close(self):
        for rk in self.ranks:
            rk.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- views of the handles' device arrays ----
    def _spectrum(self, h, nx, n1, n2, which):
        import torch
        ptr = lib().opfc_array(h, which)
        es = 8 if self.precision == FP64 else 4
        main = torch.as_tensor(_CudaArray(ptr, (n2, n1, nx, 2), self._typestr), device="cuda")
        nyq = torch.as_tensor(_CudaArray(ptr + nx * n1 * n2 * 2 * es, (n2, n1, 2), self._typestr), device="cuda")
        return main, nyq

    def _z_full(self, rk):
        """A z-slab rank's work array as one (N2/P, N1, M+1, 2) tensor (copy)."""
        import torch
        main, nyq = self._spectrum(rk.zs, self.n[0] // 2, self.n[1], self.n2loc, ARRAY_WORK)
        return torch.cat([main, nyq.unsqueeze(2)], dim=2), main, nyq

    def _kx_full(self, rk, which=ARRAY_WORK):
        import torch
        main, nyq = self._spectrum(rk.kx, self.mloc, self.n[1], self.n[2], which)
        return torch.cat([main, nyq.unsqueeze(2)], dim=2), main, nyq

    def _pass(self, h, p, mean=0.0, flags=0):
        _check(h, lib().opfc_pass(h, p, float(mean), int(flags)))

    # ---- transposes of the work arrays ----
    def _transpose_z_to_kx(self):
        import torch
        with torch.cuda.stream(self.stream):
            sends = [z_to_kx(self._z_full(rk)[0], self.P, self.mloc) for rk in self.ranks]
            recvs = self.comm.alltoall(sends)
            for rk, recv in zip(self.ranks, recvs):
                full, main, nyq = self._kx_full(rk)
                kx_from_blocks(recv, full)
                main.copy_(full[:, :, :self.mloc])
                nyq.copy_(full[:, :, self.mloc])

    def _transpose_kx_to_z(self):
        import torch
        with torch.cuda.stream(self.stream):
            sends = [kx_to_z(self._kx_full(rk)[0], self.P) for rk in self.ranks]
            recvs = self.comm.alltoall(sends)
            for rk, recv in zip(self.ranks, recvs):
                full, main, nyq = self._z_full(rk)
                z_from_blocks(recv, full, self.mloc)
                main.copy_(full[:, :, :self.n[0] // 2])
                nyq.copy_(full[:, :, self.n[0] // 2])

    def _sync(self):
        self.stream.synchronize()
        for rk in self.ranks:
            for h in (rk.zs, rk.kx):
                _check(h, lib().opfc_sync(h))

    # ---- the model ----
    def initialize(self, dt):
        for rk in self.ranks:
            _check(rk.kx, lib().opfc_initialize(rk.kx, float(dt)))

    def set_psi(self, slabs):
        """slabs[i]: this process's i-th local rank's real field, shape (N2/P, N1, N0)."""
        import torch
        sums = [math.fsum(np.asarray(s, dtype=np.float64).ravel()) for s in slabs]
        total = self.comm.allreduce_sum(sums)[0]
        self.mean = total / (self.n[0] * self.n[1] * self.n[2])
        with torch.cuda.stream(self.stream):
            for rk, s in zip(self.ranks, slabs):
                ptr = lib().opfc_array(rk.zs, ARRAY_REAL)
                real = torch.as_tensor(_CudaArray(ptr, (self.n2loc, self.n[1], self.n[0]), self._typestr), device="cuda")
                real.copy_(torch.as_tensor(np.ascontiguousarray(s), dtype=self.dtype))
        for rk in self.ranks:
            self._pass(rk.zs, PASS_XY_FORWARD)
        self._transpose_z_to_kx()
        for rk in self.ranks:  # the k = 0 slot (global rank 0's first column) stays zero
            self._pass(rk.kx, PASS_Z_FORWARD, flags=4 if rk.rank == 0 else 0)
        self._a_ready = False
        self._sync()

    def _prepare(self):
        for rk in self.ranks:
            self._pass(rk.kx, PASS_Z_INVERSE)
        self._transpose_kx_to_z()
        for rk in self.ranks:
            self._pass(rk.zs, PASS_Y_INVERSE)
        self._a_ready = True

    def step(self, n_steps=1):
        if not self._a_ready:
            self._prepare()
        for _ in range(n_steps):
            for rk in self.ranks:
                self._pass(rk.zs, PASS_X_FUSED, mean=self.mean)
                self._pass(rk.zs, PASS_Y_FORWARD)
            self._transpose_z_to_kx()
            for rk in self.ranks:
                planes = (1 if rk.rank == 0 else 0) | (2 if rk.rank == self.P - 1 else 0)
                self._pass(rk.kx, PASS_Z_UPDATE, flags=planes)
            self._transpose_kx_to_z()
            for rk in self.ranks:
                self._pass(rk.zs, PASS_Y_INVERSE)

    def sync(self):
        self._sync()

    def get_psi(self):
        """The local ranks' real z slabs (N2/P, N1, N0), FP64 host arrays."""
        import torch
        for rk in self.ranks:
            self._pass(rk.kx, PASS_Z_INVERSE_STATE)
        self._transpose_kx_to_z()
        out = []
        for rk in self.ranks:
            self._pass(rk.zs, PASS_XY_BACKWARD, mean=self.mean)
        self._sync()
        for rk in self.ranks:
            ptr = lib().opfc_array(rk.zs, ARRAY_REAL)
            real = torch.as_tensor(_CudaArray(ptr, (self.n2loc, self.n[1], self.n[0]), self._typestr), device="cuda")
            out.append(real.double().cpu().numpy())
        self._a_ready = False  # the work arrays were used for the output
        return out


class ShardedFft:
    """The sharded 3D R2C / C2R transform (the reference's IFFT contract over a
    decomposed field): forward takes each rank's real z slab and returns its kx
    slab of the half spectrum, (N2, N1, columns) complex in the reference order
    (columns [r M/P, (r+1) M/P), plus kx = M on the last rank); backward is the
    inverse with the 1/(N0 N1 N2) scaling."""

    def __init__(self, n, comm, precision=FP64, device=0):
        self._m = ShardedPfc(n, [1.0, 1.0, 1.0], comm, precision=precision, device=device)

    def close(self):
        self._m.close()

    def forward(self, slabs):
        import torch
        m = self._m
        with torch.cuda.stream(m.stream):
            for rk, s in zip(m.ranks, slabs):
                ptr = lib().opfc_array(rk.zs, ARRAY_REAL)
                real = torch.as_tensor(_CudaArray(ptr, (m.n2loc, m.n[1], m.n[0]), m._typestr), device="cuda")
                real.copy_(torch.as_tensor(np.ascontiguousarray(s), dtype=m.dtype))
        for rk in m.ranks:
            m._pass(rk.zs, PASS_XY_FORWARD)
        m._transpose_z_to_kx()
        for rk in m.ranks:
            m._pass(rk.kx, PASS_Z_FORWARD)
        m._sync()
        out = []
        for rk in m.ranks:
            full = m._kx_full(rk, ARRAY_STATE)[0].double().cpu().numpy()
            cols = m.mloc + (1 if rk.rank == m.P - 1 else 0)
            out.append(full[:, :, :cols, 0] + 1j * full[:, :, :cols, 1])
        return out

    def backward(self, spectra):
        """spectra[i]: local rank i's kx slab as returned by forward."""
        import torch
        m = self._m
        with torch.cuda.stream(m.stream):
            for rk, sp in zip(m.ranks, spectra):
                main, nyq = m._spectrum(rk.kx, m.mloc, m.n[1], m.n[2], ARRAY_STATE)
                a = np.stack([sp.real, sp.imag], axis=-1)
                main.copy_(torch.as_tensor(np.ascontiguousarray(a[:, :, :m.mloc]), dtype=m.dtype))
                if rk.rank == m.P - 1:
                    nyq.copy_(torch.as_tensor(np.ascontiguousarray(a[:, :, m.mloc]), dtype=m.dtype))
                else:
                    nyq.zero_()
        for rk in m.ranks:
            m._pass(rk.kx, PASS_Z_INVERSE_STATE)
        m._transpose_kx_to_z()
        for rk in m.ranks:
            m._pass(rk.zs, PASS_XY_BACKWARD, mean=0.0)
        m._sync()
        out = []
        for rk in m.ranks:
            ptr = lib().opfc_array(rk.zs, ARRAY_REAL)
            real = torch.as_tensor(_CudaArray(ptr, (m.n2loc, m.n[1], m.n[0]), m._typestr), device="cuda")
            out.append(real.double().cpu().numpy())
        return out
