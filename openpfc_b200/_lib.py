"""ctypes binding of libopenpfc_b200.so (C ABI in include/openpfc_b200.h).

The library is the only compute path: if it is missing or fails to load,
every call raises -- there is no CPU or PyTorch fallback.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libopenpfc_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "openpfc_b200.h")

OPFC_OK = 0
STATUS = {0: "OPFC_OK", -1: "OPFC_ERR_ARG", -2: "OPFC_ERR_SIZE", -3: "OPFC_ERR_CUDA",
          -4: "OPFC_ERR_NONFINITE", -5: "OPFC_ERR_TIMEOUT", -6: "OPFC_ERR_OOM",
          -7: "OPFC_ERR_STATE", -8: "OPFC_ERR_IO"}
FP32, FP64 = 0, 1
MODEL_PLAIN, MODEL_TUNGSTEN, MODEL_FILTERED, MODEL_ALUMINUM, MODEL_USER_ETD = 0, 1, 2, 3, 4
HOST, DEVICE = 0, 1
F32, F64 = 0, 1


class TungstenParams(ctypes.Structure):
    """Mirror of opfc_tungsten_params (tungsten_params.hpp:33-57 names)."""
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


class AluminumParams(ctypes.Structure):
    """Mirror of opfc_aluminum_params (Aluminum::params, apps/aluminumNew/Aluminum.hpp:29-82)."""
    _fields_ = [(k, ctypes.c_double) for k in
                ["n0", "n_sol", "n_vap", "T", "T0", "Bx", "T_const", "T_max", "T_min", "G_grid", "V_grid",
                 "x_initial", "m_xpos", "alpha", "alpha_farTol"]] + [("alpha_highOrd", ctypes.c_int)] + \
        [(k, ctypes.c_double) for k in
         ["tau_const", "lambda_", "stabP", "shift_u", "shift_s", "p2", "p3", "p4", "p2_bar", "p3_bar", "p4_bar",
          "q20", "q21", "q30", "q31", "q40", "q20_bar", "q21_bar", "q30_bar", "q31_bar", "q40_bar", "q2_bar",
          "q3_bar", "q4_bar", "q2_bar_L"]]


class Desc(ctypes.Structure):
    """Mirror of opfc_desc."""
    _fields_ = [("n", ctypes.c_int * 3), ("dx", ctypes.c_double * 3),
                ("origin", ctypes.c_double * 3), ("precision", ctypes.c_int),
                ("model", ctypes.c_int), ("r", ctypes.c_double),
                ("filter_alpha", ctypes.c_double), ("p2", ctypes.c_double),
                ("p3", ctypes.c_double), ("p4", ctypes.c_double),
                ("tungsten", TungstenParams), ("stream", ctypes.c_void_p),
                ("device", ctypes.c_int), ("aluminum", AluminumParams),
                ("n_global", ctypes.c_int * 3), ("kx0", ctypes.c_int)]


class OpfcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def declared_symbols() -> list[str]:
    """Every function the public header declares."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(opfc_[a-z0-9_]+)\s*\(", txt)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m openpfc_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    H = ctypes.c_void_p
    vp, sz, ci, cd = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    L.opfc_desc_default.argtypes = [ctypes.POINTER(Desc)]
    L.opfc_desc_default.restype = None
    L.opfc_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(H)]
    L.opfc_destroy.argtypes = [H]
    L.opfc_last_error.argtypes = [H]
    L.opfc_last_error.restype = ctypes.c_char_p
    L.opfc_status_string.argtypes = [ci]
    L.opfc_status_string.restype = ctypes.c_char_p
    L.opfc_initialize.argtypes = [H, cd]
    for name in ("opfc_set_psi",):
        getattr(L, name).argtypes = [H, vp, sz, ci, ci]
    for name in ("opfc_get_psi", "opfc_get_psi_hat", "opfc_get_psi_mf"):
        getattr(L, name).argtypes = [H, vp, sz, ci, ci]
    L.opfc_step.argtypes = [H, ci]
    L.opfc_sync.argtypes = [H]
    L.opfc_fft_forward.argtypes = [H, vp, vp, ci, ci]
    L.opfc_fft_backward.argtypes = [H, vp, vp, ci, ci]
    L.opfc_mass.argtypes = [H, ctypes.POINTER(cd)]
    L.opfc_free_energy.argtypes = [H, ctypes.POINTER(cd)]
    for name in ("opfc_size_inbox", "opfc_size_outbox", "opfc_allocated_bytes"):
        getattr(L, name).argtypes = [H]
        getattr(L, name).restype = sz
    L.opfc_get_stream.argtypes = [H]
    L.opfc_get_stream.restype = vp
    L.opfc_kernels_per_step.argtypes = [H]
    L.opfc_profile_step.argtypes = [H, ci, ctypes.POINTER(cd), ci]
    L.opfc_step_kernel_name.argtypes = [ci]
    L.opfc_step_kernel_name.restype = ctypes.c_char_p
    L.opfc_step_kernel_region.argtypes = [ci]
    L.opfc_step_kernel_region.restype = ctypes.c_char_p
    dp, ip = ctypes.POINTER(cd), ctypes.POINTER(ci)
    L.opfc_ic_noise.argtypes = [dp, sz, cd, cd, ctypes.c_uint64]
    L.opfc_ic_seed.argtypes = [dp, ip, dp, dp, dp, cd, cd, cd, ci]
    L.opfc_ic_seeds.argtypes = [dp, ip, dp, cd, cd, ci, cd, cd, ctypes.c_uint64]
    L.opfc_ic_seed_grid_fcc.argtypes = [dp, ip, dp, dp, ci, ci, ci, cd, cd, cd, cd, cd]
    L.opfc_ic_random_seeds.argtypes = [dp, ip, dp, dp, cd, cd]
    L.opfc_fft_forward_noalloc.argtypes = [vp, vp, ip, ci, vp]
    cp = ctypes.c_char_p
    L.opfc_format_filename.argtypes = [cp, ci, ctypes.c_char_p, sz]
    L.opfc_write_binary.argtypes = [H, cp, ci]
    L.opfc_write_binary_hat.argtypes = [H, cp, ci]
    L.opfc_read_binary.argtypes = [H, cp]
    L.opfc_write_vti.argtypes = [H, cp, ci, cp]
    L.opfc_set_time.argtypes = [H, cd, cd]
    L.opfc_set_operators.argtypes = [H, dp, dp, dp, sz]
    L.opfc_write_raw.argtypes = [cp, ip, ip, ip, dp, ci]
    L.opfc_read_raw.argtypes = [cp, ip, ip, ip, dp, ci]
    L.opfc_prepare_raw.argtypes = [cp, ip, ci]
    L.opfc_write_vti_raw.argtypes = [cp, ip, ip, ip, dp, dp, cp, dp]
    L.opfc_ensemble_create.argtypes = [ci, ctypes.POINTER(Desc), ctypes.POINTER(H)]
    L.opfc_ensemble_destroy.argtypes = [H]
    L.opfc_ensemble_last_error.argtypes = [H]
    L.opfc_ensemble_last_error.restype = ctypes.c_char_p
    L.opfc_ensemble_initialize.argtypes = [H, cd]
    L.opfc_ensemble_set_psi.argtypes = [H, ci, dp, sz]
    L.opfc_ensemble_get_psi.argtypes = [H, ci, dp, sz]
    L.opfc_ensemble_step.argtypes = [H, ci]
    L.opfc_ensemble_sync.argtypes = [H]
    L.opfc_ensemble_autotune.argtypes = [H, dp, dp, dp]
    L.opfc_ensemble_variants.argtypes = [H, ip, ip, ip]
    L.opfc_ensemble_cells.argtypes = [H]
    L.opfc_ensemble_cells.restype = sz
    L.opfc_ensemble_stream.argtypes = [H]
    L.opfc_ensemble_stream.restype = vp
    L.opfc_autotune.argtypes = [H, dp]
    L.opfc_check_bounded_wait.argtypes = [H, cd]
    L.opfc_pass.argtypes = [H, ci, cd, ci]
    L.opfc_array.argtypes = [H, ci]
    L.opfc_array.restype = vp
    L.opfc_variants.argtypes = [H, ip]
    L.opfc_set_r.argtypes = [H, cd]
    L.opfc_forward_checkpointed.argtypes = [H, ci, ci]
    L.opfc_adjoint.argtypes = [H, vp, ci, ci, vp, dp, dp]
    _lib = L
    return L


def default_desc() -> Desc:
    d = Desc()
    lib().opfc_desc_default(ctypes.byref(d))
    return d
