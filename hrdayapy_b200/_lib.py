"""ctypes binding of libhrdaya_b200.so (declarations: include/hrdaya_b200.h).

The library is the only compute path: if it is missing or no CUDA device is
present, every entry point raises instead of falling back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libhrdaya_b200.so"

HP_OK = 0
_STATUS = {1: "HP_ERR_INVALID", 2: "HP_ERR_OOM", 3: "HP_ERR_CUDA", 4: "HP_ERR_NOT_CONVERGED",
           5: "HP_ERR_STAGNATED", 6: "HP_ERR_NONFINITE", 7: "HP_ERR_TIMEOUT",
           8: "HP_ERR_UNSUPPORTED"}

HP_MAX_SITES = 8
HP_MAX_VARIANTS = 64

P = C.c_void_p


class HpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


class HpMonoDesc(C.Structure):
    _fields_ = [
        ("n_bricks", C.c_int32), ("bi", C.c_int32), ("bj", C.c_int32), ("bk", C.c_int32),
        ("anisotropic", C.c_int32),
        ("brick_nbr", P), ("tag", P), ("wface", P), ("doff", P), ("iso_coef", C.c_float),
        ("brick_variant", P), ("n_variants", C.c_int32), ("variant_gks", P), ("variant_gkr", P),
        ("n_pk", C.c_int32), ("pk_ptr", P), ("pk_idx", P), ("pk_coef", P), ("pk_stim", P),
        ("pk_variant", P),
        ("n_pmj_rows", C.c_int32), ("pmj_row", P), ("pmj_ptr", P), ("pmj_pk", P), ("pmj_coef", P),
        ("dt", C.c_double), ("Cm", C.c_double), ("v0", C.c_float), ("n_steps", C.c_int64),
        ("n_sites", C.c_int32), ("site_amp", P), ("site_on", P),
        ("n_myo", C.c_int32), ("slot_of_node", P), ("vm_every", C.c_int64),
        ("n_surf", C.c_int32), ("surf_of_slot", P), ("frame_every", C.c_int64),
        ("act_threshold", C.c_float), ("deact_threshold", C.c_float), ("max_events", C.c_int32),
        ("kernel", C.c_int32),
        ("theta", C.c_double), ("cn_tol", C.c_double), ("cn_max_iter", C.c_int32),
        ("pk_weight", C.c_float),
    ]


_lib = None


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m hrdayapy_b200.build "
                           "(there is no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    L.hp_last_error.restype = C.c_char_p
    L.hp_version.restype = C.c_char_p
    L.hp_mono_create.argtypes = [C.POINTER(HpMonoDesc), C.POINTER(P), P]
    L.hp_mono_run.argtypes = [P, C.c_int64, C.c_int32, P]
    L.hp_mono_steps_done.argtypes = [P]
    L.hp_mono_steps_done.restype = C.c_int64
    L.hp_mono_cn_stats.argtypes = [P, P, P, P, P]
    L.hp_mono_copy_vm.argtypes = [P, C.c_int64, C.c_int64, P, C.c_int32, P]
    L.hp_mono_copy_frames.argtypes = [P, C.c_int64, C.c_int64, P, P, C.c_int32, P]
    L.hp_mono_copy_events.argtypes = [P, P, P, P, P, P]
    L.hp_mono_copy_v.argtypes = [P, P, P, P]
    L.hp_mono_copy_state.argtypes = [P, P, P, P]
    L.hp_mono_destroy.argtypes = [P]
    L.hp_mono_kernel_info.argtypes = [P, P, P, P]
    _lib = L
    _declare_optional(L)
    return L


class HpTorsoDesc(C.Structure):
    _fields_ = [
        ("ni", C.c_int32), ("nj", C.c_int32), ("nk", C.c_int32), ("h_m", C.c_double),
        ("label", P), ("n_materials", C.c_int32), ("sigma", P), ("pin_row", C.c_int64),
        ("n_heart", C.c_int32), ("heart_nbr", P), ("proj", P), ("coeff", C.c_double),
        ("n_expected", C.c_double), ("n_read", C.c_int32), ("read_rows", P), ("psi", P),
    ]


class HpSolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32),
                ("rel_residual", C.c_double), ("stat", C.c_double), ("restarts", C.c_int32)]


class HpPrecondDesc(C.Structure):
    _fields_ = [("ni", C.c_int32), ("nj", C.c_int32), ("nk", C.c_int32), ("label", P),
                ("n_materials", C.c_int32), ("pin_cell", C.c_int64), ("omega", C.c_float),
                ("seed", C.c_uint64), ("init_params", P), ("sigma", P), ("h_m", C.c_double),
                ("coarse_agg", C.c_int32)]


class HpTorsoArrays(C.Structure):
    _fields_ = [("ni", C.c_int32), ("nj", C.c_int32), ("nk", C.c_int32), ("n_cells", C.c_int64),
                ("pin_cell", C.c_int64), ("label", P), ("invd", P), ("r", P), ("x", P), ("b", P)]


def _declare_optional(L):
    """Signatures of the torso entry points (include/hrdaya_b200.h)."""
    L.hp_torso_create.argtypes = [C.POINTER(HpTorsoDesc), C.POINTER(P), P]
    L.hp_torso_rows.argtypes = [P]
    L.hp_torso_rows.restype = C.c_int64
    L.hp_torso_solve_frame.argtypes = [P, P, C.c_int32, P, C.c_int32, C.c_double, C.c_int32,
                                       C.c_int32, C.POINTER(HpSolveStats), P]
    L.hp_torso_copy_solution.argtypes = [P, P, P]
    L.hp_torso_copy_rhs.argtypes = [P, P, P]
    L.hp_torso_reset.argtypes = [P]
    L.hp_torso_destroy.argtypes = [P]
    L.hp_torso_residual_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int32,
                                            C.c_double, C.c_int64, P, P, P, P]
    L.hp_precond_create.argtypes = [C.POINTER(HpPrecondDesc), C.POINTER(P), P]
    L.hp_precond_apply.argtypes = [P, P, P, P, P, C.c_int32, P]
    L.hp_precond_train_step.argtypes = [P, P, P, P, P, C.c_float, P, P]
    L.hp_precond_params.argtypes = [P, P, P, P, C.c_int32, P]
    L.hp_precond_output.argtypes = [P, P, P, P, P]
    L.hp_precond_destroy.argtypes = [P]
    L.hp_precond_coarse_info.argtypes = [P, P, P]
    L.hp_torso_arrays.argtypes = [P, C.POINTER(HpTorsoArrays)]
    L.hp_torso_solve_frame_fcg.argtypes = [P, P, P, C.c_int32, P, C.c_int32, C.c_double,
                                           C.c_int32, C.c_int32, C.c_int32,
                                           C.POINTER(HpSolveStats), P]
    L.hp_torso_train_precond.argtypes = [P, P, P, C.c_int64, C.c_int32, P, C.c_int32, C.c_int32,
                                         C.c_float, C.c_double, P, P]
    L.hp_mono_w_gather.argtypes = [P, P, C.c_int64, P, P]
    L.hp_mono_w_scatter.argtypes = [P, P, C.c_int64, P, P]
    L.hp_conv3_forward.argtypes = [P, P, P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_int32, P, P]
    L.hp_conv3_wgrad_workspace.argtypes = [C.c_int32] * 5
    L.hp_conv3_wgrad_workspace.restype = C.c_int64
    L.hp_conv3_wgrad.argtypes = [P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P,
                                 P, P, C.c_int64, P, P]


def check(status: int, what: str = ""):
    if status != HP_OK:
        msg = lib().hp_last_error().decode(errors="replace")
        if status == 1:
            raise ValueError(f"{what}: {msg}")
        raise HpError(status, f"{what}: {msg}")


def ptr(a) -> P | None:
    """Host pointer of a C-contiguous numpy array (None for None)."""
    if a is None:
        return None
    if not a.flags.c_contiguous:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(P)


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("hrdayapy_b200 needs a CUDA device (B200, sm_100a); "
                           "there is no CPU fallback")
    return torch


def current_stream():
    torch = require_cuda()
    return P(torch.cuda.current_stream().cuda_stream)
