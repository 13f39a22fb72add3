"""ctypes wrapper of the CPU FP64 oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py, always as the checker or the timed CPU
baseline.  The product package never imports this module.

Arrays follow the reference layout: real fields are numpy arrays of shape
(N2, N1, N0) (x fastest, include/openpfc/kernel/field/operations.hpp:96-103),
half spectra have shape (N2, N1, N0//2+1) complex128
(src/openpfc/runtime/cpu/fft.cpp:58-70).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_REF_OPS = os.path.join(_HERE, "_ref", "ref_ops")
_lib = None


# Where the reference source tree is mounted when this oracle is built next to
# it; OPENPFC_REFERENCE_DIR overrides it.  Only the build recipe (make ref) and
# the fixture generator read the tree; nothing on the GPU side needs it.
_DEFAULT_REFERENCE_DIR = "/root/reference"


def reference_dir():
    """The reference source tree ($OPENPFC_REFERENCE_DIR, else the default
    mount point), or None when it is absent."""
    d = os.environ.get("OPENPFC_REFERENCE_DIR") or _DEFAULT_REFERENCE_DIR
    return d if os.path.isdir(d) else None


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and _ref/ref_ops where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    d = reference_dir()
    if ref and d:
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={d}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build(ref=False)
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_r2c.argtypes = [ctypes.c_int] * 3 + [dp, dp]
        L.orc_c2r.argtypes = [ctypes.c_int] * 3 + [dp, dp]
        L.orc_fft1d.argtypes = [ctypes.c_int, dp, ctypes.c_int]
        L.orc_ops_plain.argtypes = [ip, dp, ctypes.c_double, ctypes.c_double, dp, dp]
        L.orc_filter_gauss.argtypes = [ip, dp, ctypes.c_double, dp]
        L.orc_ops_tungsten.argtypes = [ip, dp, ctypes.c_void_p, ctypes.c_double,
                                       dp, dp, dp, dp, dp]
        L.orc_tungsten_derive.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_run_plain.argtypes = [ip, dp, ctypes.c_double, ctypes.c_double, dp,
                                    ctypes.c_int, dp]
        L.orc_run_tungsten.argtypes = [ip, dp, ctypes.c_void_p, ctypes.c_double, dp,
                                       ctypes.c_int, dp]
        L.orc_run_filtered.argtypes = [ip, dp] + [ctypes.c_double] * 6 + [dp, ctypes.c_int, dp]
        cd = ctypes.c_double
        L.orc_ops_aluminum.argtypes = [ip, dp, ctypes.c_void_p, cd, dp, dp, dp, dp]
        L.orc_run_aluminum.argtypes = [ip, dp, dp, ctypes.c_void_p, cd, cd, cd, dp, ctypes.c_int, dp]
        L.orc_ic_seed_grid_fcc.argtypes = [dp, ip, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, cd, cd, cd,
                                           cd, cd]
        L.orc_ic_random_seeds.argtypes = [dp, ip, dp, dp, cd, cd]
        L.orc_sum.argtypes = [dp, ctypes.c_size_t]
        L.orc_sum.restype = ctypes.c_double
        L.orc_free_energy_plain.argtypes = [ip, dp, ctypes.c_double, dp]
        L.orc_free_energy_plain.restype = ctypes.c_double
        L.orc_ic_noise.argtypes = [ctypes.c_size_t, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_uint64, dp]
        L.orc_ic_seed_inside.argtypes = [ip, dp, dp, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, dp]
        L.orc_ic_seeds.argtypes = [ip, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_uint64, dp]
        L.orc_mt64_seed.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        L.orc_mt64_next.argtypes = [ctypes.c_void_p]
        L.orc_mt64_next.restype = ctypes.c_uint64
        L.orc_spectral_exp.argtypes = [ctypes.c_double] * 3 + [dp, dp]
        L.orc_time_plain.argtypes = [ip, dp, ctypes.c_double, ctypes.c_double, dp, ctypes.c_int]
        L.orc_time_plain.restype = ctypes.c_double
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ivec(n):
    return (ctypes.c_int * 3)(*[int(v) for v in n])


def _dvec(d):
    return (ctypes.c_double * 3)(*[float(v) for v in d])


def set_threads(t: int) -> None:
    lib().orc_set_threads(int(t))


def get_threads() -> int:
    return int(lib().orc_get_threads())


# ----------------------------------------------------------------------------
# transforms
# ----------------------------------------------------------------------------

def r2c(psi: np.ndarray) -> np.ndarray:
    """Unnormalised 3D R2C of a (N2, N1, N0) real field -> (N2, N1, N0//2+1)."""
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    n2, n1, n0 = psi.shape
    out = np.zeros((n2, n1, n0 // 2 + 1), dtype=np.complex128)
    rc = lib().orc_r2c(n0, n1, n2, _dp(psi), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0
    return out


def c2r(spec: np.ndarray, n0: int) -> np.ndarray:
    """3D C2R scaled by 1/(N0 N1 N2) (the reference's backward convention)."""
    spec = np.ascontiguousarray(spec, dtype=np.complex128)
    n2, n1, h = spec.shape
    assert h == n0 // 2 + 1
    out = np.zeros((n2, n1, n0), dtype=np.float64)
    rc = lib().orc_c2r(n0, n1, n2, spec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _dp(out))
    assert rc == 0
    return out


def fft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    y = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().orc_fft1d(len(y), y.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), sign)
    return y


# ----------------------------------------------------------------------------
# parameters and operators
# ----------------------------------------------------------------------------

class TungstenParams(ctypes.Structure):
    """Base Tungsten parameters with the defaults of
    apps/tungsten/include/tungsten/common/tungsten_params.hpp:33-57."""
    _fields_ = [("n0", ctypes.c_double), ("n_sol", ctypes.c_double),
                ("n_vap", ctypes.c_double), ("T", ctypes.c_double),
                ("T0", ctypes.c_double), ("Bx", ctypes.c_double),
                ("alpha", ctypes.c_double), ("alpha_farTol", ctypes.c_double),
                ("alpha_highOrd", ctypes.c_int), ("lambda_", ctypes.c_double),
                ("stabP", ctypes.c_double), ("shift_u", ctypes.c_double),
                ("shift_s", ctypes.c_double), ("p2", ctypes.c_double),
                ("p3", ctypes.c_double), ("p4", ctypes.c_double),
                ("q20", ctypes.c_double), ("q21", ctypes.c_double),
                ("q30", ctypes.c_double), ("q31", ctypes.c_double),
                ("q40", ctypes.c_double)]

    @classmethod
    def defaults(cls) -> "TungstenParams":
        return cls(-0.10, -0.047, -0.464, 3300.0, 156000.0, 0.8582, 0.50, 0.001, 4,
                   0.22, 0.2, 0.3341, 0.1898, 1.0, -0.5, 0.333333333, -0.0037, 1.0,
                   -12.4567, 20.0, 45.0)


class TungstenDerived(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in
                ("tau", "p2b", "p3b", "p4b", "q20b", "q21b", "q30b", "q31b",
                 "q40b", "q2b", "q3b", "q4b")]


def tungsten_derived(p: TungstenParams) -> TungstenDerived:
    d = TungstenDerived()
    lib().orc_tungsten_derive(ctypes.byref(p), ctypes.byref(d))
    return d


def _half_shape(n):
    return (n[2], n[1], n[0] // 2 + 1)


def spectral_exp(L, dt, thr=1e-12):
    e, p = ctypes.c_double(), ctypes.c_double()
    lib().orc_spectral_exp(L, dt, thr, ctypes.byref(e), ctypes.byref(p))
    return e.value, p.value


def ops_plain(n, dx, r, dt):
    opL = np.zeros(_half_shape(n))
    opN = np.zeros(_half_shape(n))
    lib().orc_ops_plain(_ivec(n), _dvec(dx), r, dt, _dp(opL), _dp(opN))
    return opL, opN


def filter_gauss(n, dx, alpha):
    chi = np.zeros(_half_shape(n))
    lib().orc_filter_gauss(_ivec(n), _dvec(dx), alpha, _dp(chi))
    return chi


def ops_tungsten(n, dx, p: TungstenParams, dt):
    outs = [np.zeros(_half_shape(n)) for _ in range(5)]
    lib().orc_ops_tungsten(_ivec(n), _dvec(dx), ctypes.byref(p), dt, *[_dp(o) for o in outs])
    fmf, expL, nw, klap, opck = outs
    return {"filterMF": fmf, "exp_Ldt": expL, "n_weight": nw, "kLap": klap, "opCk": opck}


# ----------------------------------------------------------------------------
# runs
# ----------------------------------------------------------------------------

def run_plain(psi, dx, r, dt, nsteps, norms=False):
    psi = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    nv = np.zeros(max(nsteps, 1))
    rc = lib().orc_run_plain(_ivec(n), _dvec(dx), r, dt, _dp(psi), nsteps, _dp(nv))
    assert rc == 0
    return (psi, nv[:nsteps]) if norms else psi


def time_plain(psi, dx, r, dt, nsteps):
    """Seconds for `nsteps` plain steps (tables built untimed); psi advanced in place."""
    assert psi.dtype == np.float64 and psi.flags.c_contiguous
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    t = lib().orc_time_plain(_ivec(n), _dvec(dx), r, dt, _dp(psi), nsteps)
    assert t >= 0
    return float(t)


def run_tungsten(psi, dx, p: TungstenParams, dt, nsteps, norms=False):
    psi = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    nv = np.zeros(max(nsteps, 1))
    rc = lib().orc_run_tungsten(_ivec(n), _dvec(dx), ctypes.byref(p), dt, _dp(psi), nsteps, _dp(nv))
    assert rc == 0
    return (psi, nv[:nsteps]) if norms else psi


class AluminumParams(ctypes.Structure):
    """Aluminum::params (apps/aluminumNew/Aluminum.hpp:29-82); fields not set
    stay 0 (T0 = 1), as in the reference's default-initialised struct."""
    _fields_ = [(k, ctypes.c_double) for k in
                ["n0", "n_sol", "n_vap", "T", "T0", "Bx", "T_const", "T_max", "T_min", "G_grid", "V_grid",
                 "x_initial", "m_xpos", "alpha", "alpha_farTol"]] + [("alpha_highOrd", ctypes.c_int)] + \
        [(k, ctypes.c_double) for k in
         ["tau_const", "lambda_", "stabP", "shift_u", "shift_s", "p2", "p3", "p4", "p2_bar", "p3_bar", "p4_bar",
          "q20", "q21", "q30", "q31", "q40", "q20_bar", "q21_bar", "q30_bar", "q31_bar", "q40_bar", "q2_bar",
          "q3_bar", "q4_bar", "q2_bar_L"]]

    @classmethod
    def test_case(cls):
        """The values apps/aluminumNew/aluminumTest.cpp:52-80 sets (others 0, T0 from the test)."""
        p = cls()
        p.T0 = 1.0
        for k, v in dict(n0=-0.0060, alpha=0.20, n_sol=-0.036, n_vap=-1.297, T_const=980, T_min=780,
                         T_max=1280, T0=89285.0, Bx=0.817900686921996, G_grid=0, V_grid=0, x_initial=130,
                         alpha_farTol=0.001, lambda_=0.22, stabP=0.0, shift_u=1.0, shift_s=0.0,
                         p2_bar=0.8286531831, p3_bar=-0.04204863, p4_bar=0.007533, q20_bar=0.016531729105214,
                         q21_bar=5.467, q30_bar=1.7152418049986, q31_bar=0.45, q40_bar=0.787482).items():
            setattr(p, k, v)
        p.alpha_highOrd = 0
        return p


def ops_aluminum(n, dx, p: AluminumParams, dt):
    nc = (n[0] // 2 + 1) * n[1] * n[2]
    out = [np.zeros(nc) for _ in range(4)]
    lib().orc_ops_aluminum(_ivec(n), _dvec(dx), ctypes.byref(p), dt, *[_dp(o) for o in out])
    return out  # filterMF, opL, opN, P_F


def run_aluminum(psi, dx, origin, p: AluminumParams, dt, nsteps, t0=0.0, dt_t=0.0, norms=False):
    """Aluminum steps; step s is called with time t0 + s dt_t."""
    psi = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    nv = np.zeros(max(nsteps, 1))
    rc = lib().orc_run_aluminum(_ivec(n), _dvec(dx), _dvec(origin), ctypes.byref(p), dt, t0, dt_t, _dp(psi),
                                nsteps, _dp(nv))
    assert rc == 0
    return (psi, nv[:nsteps]) if norms else psi


def ic_seed_grid_fcc(psi, dx, origin, Nx, Ny, Nz, X0, radius, amplitude, rho, rseed):
    """SeedGridFCC::apply on a pre-filled field (apps/aluminumNew/SeedGridFCC.hpp)."""
    psi = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    lib().orc_ic_seed_grid_fcc(_dp(psi), _ivec(n), _dvec(dx), _dvec(origin), int(Nx), int(Ny), int(Nz),
                               float(X0), float(radius), float(amplitude), float(rho), float(rseed))
    return psi


def ic_random_seeds(n, dx, origin, density, amplitude):
    """RandomSeeds::apply (random_seeds.hpp:54-101): 150 rotated BCC seeds from
    mt19937_64(42), 0 outside them; returns a (N2, N1, N0) field."""
    psi = np.zeros((n[2], n[1], n[0]))
    lib().orc_ic_random_seeds(_dp(psi), _ivec(n), _dvec(dx), _dvec(origin), float(density), float(amplitude))
    return psi


def run_filtered(psi, dx, r, alpha, p2, p3, p4, dt, nsteps, norms=False):
    psi = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    nv = np.zeros(max(nsteps, 1))
    rc = lib().orc_run_filtered(_ivec(n), _dvec(dx), r, alpha, p2, p3, p4, dt, _dp(psi),
                                nsteps, _dp(nv))
    assert rc == 0
    return (psi, nv[:nsteps]) if norms else psi


# ----------------------------------------------------------------------------
# diagnostics and initial conditions
# ----------------------------------------------------------------------------

def compensated_sum(a) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    return float(lib().orc_sum(_dp(a), a.size))


def free_energy_plain(psi, dx, r) -> float:
    psi = np.ascontiguousarray(psi, dtype=np.float64)
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    return float(lib().orc_free_energy_plain(_ivec(n), _dvec(dx), r, _dp(psi)))


def ic_noise(n, n0, amp, seed) -> np.ndarray:
    psi = np.zeros((n[2], n[1], n[0]))
    lib().orc_ic_noise(psi.size, n0, amp, seed, _dp(psi))
    return psi


def ic_seed_inside(psi, dx, origin, radius, rho, amp) -> np.ndarray:
    psi = np.ascontiguousarray(psi, dtype=np.float64).copy()
    n = (psi.shape[2], psi.shape[1], psi.shape[0])
    lib().orc_ic_seed_inside(_ivec(n), _dvec(dx), _dvec(origin), radius, rho, amp, _dp(psi))
    return psi


def ic_seeds(n, dx, n0, noise, nseeds, radius_cells, amp, seed) -> np.ndarray:
    psi = np.zeros((n[2], n[1], n[0]))
    lib().orc_ic_seeds(_ivec(n), _dvec(dx), n0, noise, nseeds, radius_cells, amp, seed, _dp(psi))
    return psi


class _MT(ctypes.Structure):
    _fields_ = [("mt", ctypes.c_uint64 * 312), ("mti", ctypes.c_int)]


def mt64_stream(seed: int, count: int) -> np.ndarray:
    g = _MT()
    lib().orc_mt64_seed(ctypes.byref(g), seed)
    return np.array([lib().orc_mt64_next(ctypes.byref(g)) for _ in range(count)], dtype=np.uint64)


# ----------------------------------------------------------------------------
# the reference's own operator code (only where the reference tree exists)
# ----------------------------------------------------------------------------

_REF_SEEDS = os.path.join(_HERE, "_ref", "ref_seeds")


def ref_random_seeds(n, dx, origin, density, amplitude, tmpdir):
    """Run _ref/ref_seeds (the reference's Seed class compiled in place)."""
    path = os.path.join(tmpdir, f"ref_seeds_{n[0]}_{n[1]}_{n[2]}.bin")
    args = [str(int(v)) for v in n] + [repr(float(v)) for v in dx] + [repr(float(v)) for v in origin]
    subprocess.run([_REF_SEEDS] + args + [repr(float(density)), repr(float(amplitude)), path], check=True)
    return np.fromfile(path, dtype=np.float64).reshape(n[2], n[1], n[0])


def ref_ops_available() -> bool:
    return os.path.exists(_REF_OPS)


def ref_ops(n, dx, dt, tmpdir):
    """Run _ref/ref_ops (reference headers compiled in place) and parse its tables."""
    path = os.path.join(tmpdir, f"ref_ops_{n[0]}_{n[1]}_{n[2]}.bin")
    subprocess.run([_REF_OPS, str(n[0]), str(n[1]), str(n[2]), repr(float(dx)),
                    repr(float(dt)), path], check=True)
    raw = np.fromfile(path, dtype=np.float64)
    nc = (n[0] // 2 + 1) * n[1] * n[2]
    derived = raw[:12]
    t = raw[12:].reshape(3, nc)
    shp = _half_shape(n)
    return {"derived": derived, "filterMF": t[0].reshape(shp),
            "exp_Ldt": t[1].reshape(shp), "n_weight": t[2].reshape(shp)}

