"""ctypes binding of the C ABI in include/trajsparsenufft.h.

The shared library is built in-tree (``python -m trajsparsenufft_b200.build``).
There is no fallback: if the library is missing or fails to load, every entry
point raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtrajsparsenufft.so"

STATUS = {
    0: "OK", 1: "IO", 2: "FORMAT", 3: "SHAPE", 4: "NONFINITE", 5: "CURVATURE", 6: "TIMEOUT",
    7: "CUDA", 8: "ARG", 9: "UNSUPPORTED", 10: "NOMEM",
}

PLANNER = {"optimized": 0, "fast": 1, "search": 2}
POLICY = {"trajectory": 0, "morton": 1, "overlap": 2, "packing256": 3}
ILLEGAL = {"split24": 0, "csr_residual": 1}
VIEW = {"G": 0, "G_T": 1}
FLAG_REFERENCE_LAYOUT = 1
FLAG_REFERENCE_STEPS = 2
CG_STEP_PARTS = 296  # TSN_CG_STEP_PARTS
STAGES = ("fwd_rows", "fwd_cols", "interp_fwd", "interp_adj", "inv_cols", "inv_rows", "cg_update", "fwd_mid",
          "inv_mid")

EXPORTED = (
    "tsn_version", "tsn_get_last_error_string", "tsn_plan_desc_default", "tsn_kb_interpolation_csr",
    "tsn_kb_deapodization", "tsn_kb_weights_csr3", "tsn_kb_deapodization3", "tsn_pack_csr_to_dirs", "tsn_pack_view_tiles", "tsn_export_view_dir",
    "tsn_plan_create_from_pack", "tsn_plan_create_from_trajectory", "tsn_plan_destroy", "tsn_plan_get_info",
    "tsn_forward", "tsn_adjoint", "tsn_forward_reference", "tsn_adjoint_reference", "tsn_normal", "tsn_rdot", "tsn_cg_step", "tsn_cg_adjoint_step", "tsn_cg_adjoint_finish", "tsn_cg_sense", "tsn_cg_sense_ex", "tsn_batch_create", "tsn_batch_destroy", "tsn_batch_cg_sense",
    "tsn_fft_forward_panel", "tsn_fft_adjoint_image", "tsn_profile_stages", "tsn_fft_adjoint_image_static",
    "tsn_interp_component",
)


class TsnError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.kind = STATUS.get(status, str(status))


class PlanDesc(C.Structure):
    _fields_ = [
        ("im_size", C.c_int32), ("grid_size", C.c_int32), ("coils", C.c_int32), ("kernel_width", C.c_int32),
        ("planner", C.c_int32), ("policy", C.c_int32), ("seed", C.c_uint64), ("threads", C.c_int32),
        ("flags", C.c_int32), ("interp", C.c_int32), ("device", C.c_int32), ("dims", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class PlanInfo(C.Structure):
    _fields_ = [
        ("samples", C.c_int64), ("im_size", C.c_int32), ("grid_size", C.c_int32), ("coils", C.c_int32),
        ("kernel_width", C.c_int32), ("components", C.c_int32),
        ("groups", C.c_int64 * 2), ("tiles", C.c_int64 * 2), ("active_rows", C.c_int64 * 2),
        ("nnz", C.c_int64 * 2), ("pack_bytes", C.c_int64 * 2), ("workspace_bytes", C.c_int64),
        ("plan_seconds", C.c_double), ("interp", C.c_int32), ("dims", C.c_int32), ("device_error", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class CgOptions(C.Structure):
    _fields_ = [("reliable_update_period", C.c_int32), ("reliable_update_direction", C.c_int32),
                ("scheduled_reference_period", C.c_int32), ("reserved0", C.c_int32),
                ("reference_steps", C.c_uint64), ("reserved", C.c_int32 * 2)]


class CgStatus(C.Structure):
    _fields_ = [
        ("completed_iterations", C.c_int32), ("positive_curvature", C.c_int32), ("finite", C.c_int32),
        ("timeout", C.c_int32), ("residual0", C.c_double), ("residual_final", C.c_double),
    ]


_LIB = None

P = C.c_void_p
I32, I64, U64, F32, F64 = C.c_int32, C.c_int64, C.c_uint64, C.c_float, C.c_double
PI64, PF64, PF32, PI32, PU8 = (C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_float),
                               C.POINTER(C.c_int32), C.POINTER(C.c_uint8))


def lib() -> C.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH.name} is not built; run `python -m trajsparsenufft_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "tsn_version": (C.c_char_p, []),
        "tsn_get_last_error_string": (C.c_char_p, []),
        "tsn_plan_desc_default": (C.c_int, [C.POINTER(PlanDesc)]),
        "tsn_kb_interpolation_csr": (C.c_int, [PF32, I64, I32, I32, I32, PI64, PI64, PF64, PF64, PI64]),
        "tsn_kb_deapodization": (C.c_int, [I32, I32, I32, PF64]),
        "tsn_kb_weights_csr3": (C.c_int, [PF32, I64, I32, I32, I32, PI64, PI64, PF64, PI64]),
        "tsn_kb_deapodization3": (C.c_int, [I32, I32, I32, PF64]),
        "tsn_pack_csr_to_dirs": (C.c_int, [PI64, PI64, PF64, PF64, I64, I32, PF32, I32, I32, I32, U64, I32,
                                           C.c_char_p]),
        "tsn_pack_view_tiles": (C.c_int, [PI64, PI64, PF64, PI64, PF64, I64, I64, I64, I32, I32, I32, U64, I32,
                                          PI64, PI32, PI32, PF64, PU8]),
        "tsn_export_view_dir": (C.c_int, [PI64, PI64, PF64, PI64, PF64, I64, I64, I64, I32, I32, U64, I32, I32,
                                          C.c_char_p]),
        "tsn_plan_create_from_pack": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, PF32,
                                                C.POINTER(PlanDesc), C.POINTER(P)]),
        "tsn_plan_create_from_trajectory": (C.c_int, [PF32, I64, C.POINTER(PlanDesc), C.POINTER(P)]),
        "tsn_plan_destroy": (C.c_int, [P]),
        "tsn_plan_get_info": (C.c_int, [P, C.POINTER(PlanInfo)]),
        "tsn_forward": (C.c_int, [P, P, P, P, P]),
        "tsn_adjoint": (C.c_int, [P, P, P, P, P]),
        "tsn_forward_reference": (C.c_int, [P, P, P, P, P]),
        "tsn_normal": (C.c_int, [P, P, P, P, C.c_float, P, P, P, P, C.c_int32, P]),
        "tsn_rdot": (C.c_int, [P, P, P, C.c_int64, P, P]),
        "tsn_cg_step": (C.c_int, [P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P, P]),
        "tsn_cg_adjoint_step": (C.c_int, [P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P, P, P, P]),
        "tsn_cg_adjoint_finish": (C.c_int, [P, C.c_int64, C.c_int32, P, P, P, P, P, P, P, P]),
        "tsn_adjoint_reference": (C.c_int, [P, P, P, P, P]),
        "tsn_cg_sense": (C.c_int, [P, P, P, P, F32, F32, I32, P, PF64, C.POINTER(CgStatus), P]),
        "tsn_cg_sense_ex": (C.c_int, [P, P, P, P, F32, F32, I32, C.POINTER(CgOptions), P, PF64,
                                      C.POINTER(CgStatus), P]),
        "tsn_batch_create": (C.c_int, [C.POINTER(P), I32, I32, C.POINTER(P)]),
        "tsn_batch_destroy": (C.c_int, [P]),
        "tsn_batch_cg_sense": (C.c_int, [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), F32, F32, I32,
                                         C.POINTER(P), C.POINTER(CgStatus), P]),
        "tsn_fft_forward_panel": (C.c_int, [P, P, P, P, PF32, P]),
        "tsn_profile_stages": (C.c_int, [P, P, P, I32, PF64, P]),
        "tsn_fft_adjoint_image_static": (C.c_int, [I32, I32, I32, I32, P, P, P, P, P]),
        "tsn_fft_adjoint_image": (C.c_int, [P, P, P, P, P]),
        "tsn_interp_component": (C.c_int, [P, I32, I32, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def check(status: int) -> None:
    if status != 0:
        raise TsnError(status, lib().tsn_get_last_error_string().decode(errors="replace"))


def ptr(array, ctype):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if array is None:
        return None
    return array.ctypes.data_as(C.POINTER(ctype))
