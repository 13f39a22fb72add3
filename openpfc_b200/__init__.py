"""openpfc_b200 -- B200-native spectral PFC time step behind OpenPFC's API.

The compute path is libopenpfc_b200.so (hand-written sm_100a kernels, C ABI in
include/openpfc_b200.h).  This module is the Python mirror of the reference's
host interface for that path:

  * :class:`B200Fft`   -- pfc::fft::IFFT (include/openpfc/kernel/fft/fft_interface.hpp:40-83)
  * :class:`PfcB200`   -- the plain conserved PFC model
                          (docs/api/examples/10_complete_pfc_model.cpp:62-214)
  * :class:`TungstenB200` -- the Tungsten model (apps/tungsten/include/tungsten/
                          cpu/tungsten_model.hpp:123-380), params as TungstenParams
  * :class:`FilteredB200` -- Gaussian mean-field filter + polynomial of psi_MF

Errors follow the reference: size contracts raise ValueError (the reference's
std::invalid_argument), everything else raises RuntimeError.  Host arrays are
numpy (x fastest: shape (N2, N1, N0)); device arrays are torch CUDA tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (DEVICE, F32, F64, FP32, FP64, HOST, MODEL_ALUMINUM, MODEL_FILTERED, MODEL_PLAIN,
                   MODEL_TUNGSTEN, MODEL_USER_ETD, AluminumParams, Desc, OpfcError, TungstenParams,
                   default_desc, lib)

__all__ = ["B200Fft", "PfcB200", "TungstenB200", "FilteredB200", "AluminumB200", "AluminumParams", "EtdB200", "Desc",
           "TungstenParams",
           "OpfcError", "default_desc", "lib", "FP32", "FP64"]


def _check(h, rc: int):
    if rc != 0:
        msg = lib().opfc_last_error(h).decode() if h else ""
        if rc == -2:
            raise ValueError(f"OPFC_ERR_SIZE: {msg}")
        raise OpfcError(rc, msg)


def _buf(arr, writable: bool = False):
    """(pointer, count, dtype code, location) of a numpy array or torch tensor."""
    if isinstance(arr, np.ndarray):
        if not arr.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        if arr.dtype == np.float64:
            dt = F64
        elif arr.dtype == np.float32:
            dt = F32
        else:
            raise ValueError(f"unsupported dtype {arr.dtype}")
        return ctypes.c_void_p(arr.ctypes.data), arr.size, dt, HOST
    import torch  # device buffers are torch tensors
    if isinstance(arr, torch.Tensor):
        if not arr.is_contiguous():
            raise ValueError("tensor must be contiguous")
        if arr.dtype == torch.float64:
            dt = F64
        elif arr.dtype == torch.float32:
            dt = F32
        else:
            raise ValueError(f"unsupported dtype {arr.dtype}")
        loc = DEVICE if arr.is_cuda else HOST
        return ctypes.c_void_p(arr.data_ptr()), arr.numel(), dt, loc
    raise TypeError(f"unsupported buffer type {type(arr)}")


class _Handle:
    def __init__(self, desc: Desc):
        self._h = ctypes.c_void_p()
        self.desc = desc
        _check(None, lib().opfc_create(ctypes.byref(desc), ctypes.byref(self._h)))
        self.shape = (desc.n[2], desc.n[1], desc.n[0])
        self.half_shape = (desc.n[2], desc.n[1], desc.n[0] // 2 + 1)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().opfc_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def size_inbox(self) -> int:
        return int(lib().opfc_size_inbox(self._h))

    def size_outbox(self) -> int:
        return int(lib().opfc_size_outbox(self._h))

    def get_allocated_memory_bytes(self) -> int:
        return int(lib().opfc_allocated_bytes(self._h))

    @property
    def stream(self) -> int:
        return int(lib().opfc_get_stream(self._h) or 0)

    @property
    def real_dtype(self):
        return np.float64 if self.desc.precision == FP64 else np.float32


class B200Fft(_Handle):
    """pfc::fft::IFFT on one B200: forward R2C unnormalised, backward C2R scaled
    by 1/(N0 N1 N2) (fft_heffte_backend.hpp:216,243).  Sizes are checked like the
    reference (fft_heffte_backend.hpp:151-156)."""

    def __init__(self, n, dx=(1.0, 1.0, 1.0), precision: int = FP64, device: int = 0):
        d = default_desc()
        for a in range(3):
            d.n[a] = int(n[a])
            d.dx[a] = float(dx[a])
        d.precision = precision
        d.device = device
        super().__init__(d)
        self._fft_time = 0.0

    def forward(self, inp, out=None):
        if out is None:
            out = np.zeros(self.half_shape, dtype=np.complex128)
        ob = out.view(np.float64) if isinstance(out, np.ndarray) and out.dtype == np.complex128 else \
            (out.view(np.float32) if isinstance(out, np.ndarray) and out.dtype == np.complex64 else out)
        ip, icnt, idt, iloc = _buf(inp)
        op, ocnt, odt, oloc = _buf(ob)
        if icnt != self.size_inbox() or ocnt != 2 * self.size_outbox():
            raise ValueError(f"FFT forward: expected {self.size_inbox()} reals in and "
                             f"{self.size_outbox()} complex out, got {icnt} and {ocnt // 2}")
        if idt != odt or iloc != oloc:
            raise ValueError("input and output must share dtype and location")
        _check(self._h, lib().opfc_fft_forward(self._h, ip, op, idt, iloc))
        return out

    def backward(self, inp, out=None):
        if out is None:
            out = np.zeros(self.shape, dtype=np.float64)
        ib = inp.view(np.float64) if isinstance(inp, np.ndarray) and inp.dtype == np.complex128 else \
            (inp.view(np.float32) if isinstance(inp, np.ndarray) and inp.dtype == np.complex64 else inp)
        ip, icnt, idt, iloc = _buf(np.ascontiguousarray(ib) if isinstance(ib, np.ndarray) else ib)
        op, ocnt, odt, oloc = _buf(out)
        if icnt != 2 * self.size_outbox() or ocnt != self.size_inbox():
            raise ValueError(f"FFT backward: expected {self.size_outbox()} complex in and "
                             f"{self.size_inbox()} reals out, got {icnt // 2} and {ocnt}")
        if idt != odt or iloc != oloc:
            raise ValueError("input and output must share dtype and location")
        _check(self._h, lib().opfc_fft_backward(self._h, ip, op, idt, iloc))
        return out

    def reset_fft_time(self):
        self._fft_time = 0.0

    def get_fft_time(self) -> float:
        return self._fft_time


class _ModelBase(_Handle):
    def initialize(self, dt: float):
        _check(self._h, lib().opfc_initialize(self._h, float(dt)))

    def set_psi(self, psi):
        p, cnt, dt, loc = _buf(psi)
        _check(self._h, lib().opfc_set_psi(self._h, p, cnt, dt, loc))

    def get_psi(self, out=None):
        if out is None:
            out = np.zeros(self.shape, dtype=np.float64)
        p, cnt, dt, loc = _buf(out)
        _check(self._h, lib().opfc_get_psi(self._h, p, cnt, dt, loc))
        return out

    def get_psi_mf(self, out=None):
        if out is None:
            out = np.zeros(self.shape, dtype=np.float64)
        p, cnt, dt, loc = _buf(out)
        _check(self._h, lib().opfc_get_psi_mf(self._h, p, cnt, dt, loc))
        return out

    def get_psi_hat(self, out=None):
        if out is None:
            out = np.zeros(self.half_shape, dtype=np.complex128)
        ob = out.view(np.float64) if out.dtype == np.complex128 else out.view(np.float32)
        p, cnt, dt, loc = _buf(ob)
        _check(self._h, lib().opfc_get_psi_hat(self._h, p, cnt // 2, dt, loc))
        return out

    def step(self, n_steps: int = 1):
        """Advance n_steps steps (asynchronous; see :meth:`sync`)."""
        _check(self._h, lib().opfc_step(self._h, int(n_steps)))

    def sync(self):
        _check(self._h, lib().opfc_sync(self._h))

    def mass(self) -> float:
        v = ctypes.c_double()
        _check(self._h, lib().opfc_mass(self._h, ctypes.byref(v)))
        return v.value

    def free_energy(self) -> float:
        v = ctypes.c_double()
        _check(self._h, lib().opfc_free_energy(self._h, ctypes.byref(v)))
        return v.value

    # on-disk formats of the reference (BinaryWriter / FileReader / VTKWriter)
    def write_binary(self, pattern: str, increment: int = 0):
        """psi as raw FP64, x fastest, no header; file format_with_number(pattern, increment)."""
        _check(self._h, lib().opfc_write_binary(self._h, pattern.encode(), int(increment)))

    def write_binary_hat(self, pattern: str, increment: int = 0):
        """psi_hat, reference layout, raw interleaved complex FP64."""
        _check(self._h, lib().opfc_write_binary_hat(self._h, pattern.encode(), int(increment)))

    def read_binary(self, filename: str):
        """Set the state from a raw FP64 psi file (FileReader initial condition)."""
        _check(self._h, lib().opfc_read_binary(self._h, filename.encode()))

    def write_vti(self, pattern: str, increment: int = 0, field_name: str = "Field"):
        """psi as VTK XML ImageData (.vti), Float64, appended raw."""
        _check(self._h, lib().opfc_write_vti(self._h, pattern.encode(), int(increment), field_name.encode()))

    def kernels_per_step(self) -> int:
        return int(lib().opfc_kernels_per_step(self._h))

    def autotune(self) -> dict:
        """Time every kernel variant of each pass, keep the fastest (cached per
        device); returns ms per launch by variant.  Set the field afterwards."""
        names = ["y.pipelined", "y.direct", "y.narrow", "y.pingpong", "y.direct_e32", "x.pipelined", "x.direct",
                 "x.no_square",
                 "x.square_direct", "x.square_direct_prefetch",
                 "z.tables", "z.radial", "z.direct", "z.computed", "z.direct_computed", "z.computed_pingpong",
                 "z.folded_pingpong", "z.direct_folded", "z.folded", "z.folded_wide"]
        ms = (ctypes.c_double * len(names))()
        _check(self._h, lib().opfc_autotune(self._h, ms))
        return dict(zip(names, list(ms)))

    def forward_checkpointed(self, n_steps: int, K: int = 20):
        """Advance n_steps, keeping a snapshot every K steps for :meth:`adjoint`."""
        _check(self._h, lib().opfc_forward_checkpointed(self._h, int(n_steps), int(K)))

    def adjoint(self, grad_psi_T, out=None):
        """(dLoss/dpsi0, dLoss/dr, dLoss/dn0) for dLoss/dpsi_T = grad_psi_T; dLoss/dr
        is NaN for models without r (Tungsten, Aluminum, caller-supplied operators)."""
        if out is None:
            out = np.zeros(self.shape, dtype=np.float64) if isinstance(grad_psi_T, np.ndarray) \
                else grad_psi_T.new_zeros(grad_psi_T.shape)
        gp, gc, gdt, gloc = _buf(grad_psi_T)
        op, oc, odt, oloc = _buf(out)
        if gc != self.size_inbox() or oc != gc or gdt != odt or gloc != oloc:
            raise ValueError("gradient buffers must be N0*N1*N2 values of one dtype and location")
        gr, gn = ctypes.c_double(), ctypes.c_double()
        _check(self._h, lib().opfc_adjoint(self._h, gp, gdt, gloc, op, ctypes.byref(gr), ctypes.byref(gn)))
        return out, gr.value, gn.value

    def variants(self) -> tuple:
        v = (ctypes.c_int * 3)()
        _check(self._h, lib().opfc_variants(self._h, v))
        return tuple(v)

    def profile_step(self, reps: int = 10) -> dict:
        """Mean ms per launch of each kernel of the step, timed alone with CUDA
        events on the handle's stream.  Leaves the field undefined."""
        ms = (ctypes.c_double * 8)()
        n = lib().opfc_profile_step(self._h, int(reps), ms, 8)
        if n < 0:
            _check(self._h, n)
        return {lib().opfc_step_kernel_name(k).decode(): ms[k] for k in range(n)}


def _geom(d: Desc, n, dx, origin, precision, device, stream):
    for a in range(3):
        d.n[a] = int(n[a])
        d.dx[a] = float(dx[a])
        d.origin[a] = float(origin[a]) if origin is not None else 0.0
    d.precision = precision
    d.device = device
    d.stream = stream


class PfcB200(_ModelBase):
    """Plain conserved PFC: L(k) = -k^2 (r + (1-k^2)^2), opL = exp(L dt),
    opN = (opL - 1)/L (-k^2) (10_complete_pfc_model.cpp:166-213); N = psi^3."""

    def __init__(self, n, dx, r: float = -0.25, precision: int = FP32, device: int = 0,
                 origin=None, stream=None):
        d = default_desc()
        _geom(d, n, dx, origin, precision, device, stream)
        d.model = MODEL_PLAIN
        d.r = float(r)
        super().__init__(d)

    def set_r(self, r: float):
        _check(self._h, lib().opfc_set_r(self._h, float(r)))
        self.desc.r = float(r)


class FilteredB200(_ModelBase):
    """Mean-field-filtered PFC: psi_MF = F^-1[exp(-k^2/(2 alpha^2)) psi_hat],
    N = p2 psi_MF^2/2 + p3 psi_MF^3/3 + p4 psi_MF^4/4, plain opL/opN at r."""

    def __init__(self, n, dx, r=-0.3, alpha=0.5, p2=-0.1, p3=-0.5, p4=0.3,
                 precision: int = FP32, device: int = 0, origin=None, stream=None):
        d = default_desc()
        _geom(d, n, dx, origin, precision, device, stream)
        d.model = MODEL_FILTERED
        d.r, d.filter_alpha, d.p2, d.p3, d.p4 = float(r), float(alpha), float(p2), float(p3), float(p4)
        super().__init__(d)

    def set_r(self, r: float):
        _check(self._h, lib().opfc_set_r(self._h, float(r)))
        self.desc.r = float(r)


class TungstenB200(_ModelBase):
    """Tungsten model; ``params`` is a TungstenParams (defaults of tungsten_params.hpp)."""

    def __init__(self, n, dx, params: TungstenParams | None = None, precision: int = FP64,
                 device: int = 0, origin=None, stream=None):
        d = default_desc()
        _geom(d, n, dx, origin, precision, device, stream)
        d.model = MODEL_TUNGSTEN
        if params is not None:
            d.tungsten = params
        super().__init__(d)


class AluminumB200(_ModelBase):
    """Aluminum PFC variant (apps/aluminumNew/Aluminum.hpp): Tungsten-form step
    with the two-Gaussian correlation peak P_F; ``params`` is an AluminumParams
    (fields the caller leaves unset stay 0, T0 = 1, as in the reference).  With
    G_grid != 0 the moving temperature T_var(x, t) acts: set_time(t, dt_t) gives
    the time of the next step (then advanced by dt_t per step)."""

    def set_time(self, t: float, dt_per_step: float):
        _check(self._h, lib().opfc_set_time(self._h, float(t), float(dt_per_step)))

    def __init__(self, n, dx, params: AluminumParams | None = None, precision: int = FP64,
                 device: int = 0, origin=None, stream=None):
        d = default_desc()
        _geom(d, n, dx, origin, precision, device, stream)
        d.model = MODEL_ALUMINUM
        if params is not None:
            d.aluminum = params
        super().__init__(d)


class EtdB200(_ModelBase):
    """Caller-supplied ETD1 operators on the fused passes (the GPU backend of the
    reference's Etd1Stepper, include/openpfc/kernel/simulation/steppers/etd1.hpp):
    psi_hat <- exp_Ldt psi_hat + n_weight F[N], N = p2 v^2/2 + p3 v^3/3 + p4 v^4/4
    of v = F^-1[chi psi_hat].  set_operators() takes arrays of the reference's
    half-spectrum shape (N2, N1, N0//2+1); k = 0 must conserve the mean."""

    def __init__(self, n, dx, p2: float = 0.0, p3: float = 0.0, p4: float = 0.0, precision: int = FP64,
                 device: int = 0, origin=None, stream=None):
        d = default_desc()
        _geom(d, n, dx, origin, precision, device, stream)
        d.model = MODEL_USER_ETD
        d.p2, d.p3, d.p4 = float(p2), float(p3), float(p4)
        self._nc = (int(n[0]) // 2 + 1) * int(n[1]) * int(n[2])
        super().__init__(d)

    def set_operators(self, exp_Ldt, n_weight, chi=None):
        a = np.ascontiguousarray(exp_Ldt, dtype=np.float64).ravel()
        b = np.ascontiguousarray(n_weight, dtype=np.float64).ravel()
        c = None if chi is None else np.ascontiguousarray(chi, dtype=np.float64).ravel()
        dp = ctypes.POINTER(ctypes.c_double)
        _check(self._h, lib().opfc_set_operators(self._h, a.ctypes.data_as(dp), b.ctypes.data_as(dp),
                                                 None if c is None else c.ctypes.data_as(dp), a.size))


# ---------------------------------------------------------------------------
# file names (pfc::utils::format_with_number)
# ---------------------------------------------------------------------------

def format_with_number(pattern: str, increment: int) -> str:
    """A pattern without '%' unchanged; else exactly one %d (flags -+ 0, width)
    replaced by the increment; anything else raises ValueError."""
    out = ctypes.create_string_buffer(4096)
    rc = lib().opfc_format_filename(pattern.encode(), int(increment), out, len(out))
    if rc == -1:
        raise ValueError(f"invalid filename pattern {pattern!r}")
    if rc != 0:
        raise RuntimeError(f"opfc_format_filename failed ({rc})")
    return out.value.decode()


# ---------------------------------------------------------------------------
# initial conditions (host-side set-up, libopenpfc_b200.so)
# ---------------------------------------------------------------------------

def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i3(v):
    return (ctypes.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return (ctypes.c_double * 3)(*[float(x) for x in v])


def ic_noise(n, n0: float, amp: float, seed: int) -> np.ndarray:
    """psi = n0 + U(-amp, amp) per cell (x fastest), std::mt19937_64(seed)."""
    psi = np.empty((n[2], n[1], n[0]), dtype=np.float64)
    _check(None, lib().opfc_ic_noise(_dp(psi), psi.size, n0, amp, seed))
    return psi


def ic_seed(psi: np.ndarray, dx, origin, center, radius, rho, amp, outside_zero=False):
    """One-mode BCC seed (single_seed.hpp); modifies and returns psi."""
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    assert psi.dtype == np.float64 and psi.flags.c_contiguous
    _check(None, lib().opfc_ic_seed(_dp(psi), _i3(n), _d3(dx), _d3(origin), _d3(center), radius,
                                    rho, amp, int(outside_zero)))
    return psi


def ic_seed_grid_fcc(psi: np.ndarray, dx, origin, Nx, Ny, Nz, X0, radius, amplitude, rho, rseed) -> np.ndarray:
    """SeedGridFCC (apps/aluminumNew/SeedGridFCC.hpp) applied to a copy of psi."""
    out = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (out.shape[2], out.shape[1], out.shape[0])
    rc = lib().opfc_ic_seed_grid_fcc(_dp(out), _i3(n), _d3(dx), _d3(origin), int(Nx), int(Ny), int(Nz),
                                     float(X0), float(radius), float(amplitude), float(rho), float(rseed))
    if rc != 0:
        raise ValueError(f"opfc_ic_seed_grid_fcc: {rc}")
    return out


def ic_random_seeds(n, dx, origin, density, amplitude) -> np.ndarray:
    """RandomSeeds (include/openpfc/kernel/simulation/initial_conditions/
    random_seeds.hpp): 150 rotated one-mode BCC seeds of radius 20 drawn from
    std::mt19937_64(42) in the reference's fixed box, 0 outside them; returns a
    (N2, N1, N0) field."""
    out = np.zeros((n[2], n[1], n[0]))
    _check(None, lib().opfc_ic_random_seeds(_dp(out), _i3(n), _d3(dx), _d3(origin), float(density),
                                            float(amplitude)))
    return out


def ic_seeds(n, dx, n0, noise, nseeds, radius_cells, amp, seed) -> np.ndarray:
    """Noisy liquid with `nseeds` seeded BCC spheres (see opfc_ic_seeds)."""
    psi = np.empty((n[2], n[1], n[0]), dtype=np.float64)
    _check(None, lib().opfc_ic_seeds(_dp(psi), _i3(n), _d3(dx), n0, noise, nseeds, radius_cells,
                                     amp, seed))
    return psi


# ---------------------------------------------------------------------------
# uneven-size ensembles (opfc_ensemble_*)
# ---------------------------------------------------------------------------

class Ensemble:
    """Independent plain-PFC fields of different sizes and parameters advanced
    together: one persistent kernel per stage, the step loop in one CUDA graph.

    members: sequence of dicts with keys n (N0, N1, N2), dx (3 values), r."""

    def __init__(self, members, precision: int = FP32, device: int = 0):
        descs = (Desc * len(members))()
        for i, mb in enumerate(members):
            lib().opfc_desc_default(ctypes.byref(descs[i]))
            _geom(descs[i], mb["n"], mb["dx"], None, precision, device, None)
            descs[i].model = MODEL_PLAIN
            descs[i].r = float(mb["r"])
        self._h = ctypes.c_void_p()
        rc = lib().opfc_ensemble_create(len(members), descs, ctypes.byref(self._h))
        if rc != 0:
            if rc == -2:
                raise ValueError("OPFC_ERR_SIZE: unsupported member size")
            raise OpfcError(rc, "opfc_ensemble_create")
        self.members = [dict(m) for m in members]
        self.shapes = [(m["n"][2], m["n"][1], m["n"][0]) for m in members]

    def _check(self, rc):
        if rc != 0:
            msg = lib().opfc_ensemble_last_error(self._h).decode()
            if rc == -2:
                raise ValueError(f"OPFC_ERR_SIZE: {msg}")
            raise OpfcError(rc, msg)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().opfc_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def initialize(self, dt: float):
        self._check(lib().opfc_ensemble_initialize(self._h, float(dt)))

    def set_psi(self, i: int, psi: np.ndarray):
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        self._check(lib().opfc_ensemble_set_psi(self._h, int(i), _dp(psi), psi.size))

    def get_psi(self, i: int) -> np.ndarray:
        out = np.empty(self.shapes[i], dtype=np.float64)
        self._check(lib().opfc_ensemble_get_psi(self._h, int(i), _dp(out), out.size))
        return out

    def step(self, n_steps: int):
        self._check(lib().opfc_ensemble_step(self._h, int(n_steps)))

    def sync(self):
        self._check(lib().opfc_ensemble_sync(self._h))

    def autotune(self):
        """Time the tile-shape / occupancy variants of the y, x and z-update
        stages, keep the fastest of each; states must be set again.  Returns
        the milliseconds per variant: (y, x, z update)."""
        mc, mx, mu = (ctypes.c_double * 6)(), (ctypes.c_double * 6)(), (ctypes.c_double * 6)()
        self._check(lib().opfc_ensemble_autotune(self._h, mc, mx, mu))
        return list(mc), list(mx), list(mu)

    def variants(self):
        """Chosen variants (y passes, x pass, z update)."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(lib().opfc_ensemble_variants(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    @property
    def cells(self) -> int:
        return int(lib().opfc_ensemble_cells(self._h))

    @property
    def stream(self) -> int:
        return int(lib().opfc_ensemble_stream(self._h) or 0)
