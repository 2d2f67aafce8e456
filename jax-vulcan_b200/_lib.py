"""ctypes binding of ``libvulcan_b200.so`` (the C-ABI in include/vulcan_b200.h).

There is no fallback: if the library is missing the import of a compute
function raises. Device buffers are passed as raw pointers of torch tensors on
the current CUDA stream.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvulcan_b200.so")

VB_USE_VM_MOL = 1
VB_USE_SETTLING = 2
VB_USE_TOPFLUX = 4
VB_USE_BOTFLUX = 8
VB_MAX_NI = 128

STATUS_BITS = {1: "zero pivot", 2: "non-finite", 4: "refinement stall", 8: "watchdog"}

_p = C.c_void_p
_i = C.c_int
_i32 = C.c_int32
_sz = C.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "vb_last_error": (C.c_char_p, []),
    "vb_version": (_i, []),
    "vb_net_create": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, C.POINTER(_p)]),
    "vb_net_destroy": (_i, [_p]),
    "vb_net_device_bytes": (_sz, [_p]),
    "vb_net_set_tuning": (_i, [_p, _p]),
    "vb_net_get_tuning": (_i, [_p, _p]),
    "vb_ros2_workspace_bytes": (_sz, [_i, _i, _i, _p]),
    "vb_ros2_assembly_bytes": (_sz, [_p, _i, _i]),
    "vb_ros2_step": (_i, [_p, _i, _i, _p, _p, _p, _p, _p, _i32, _p, _p, _p, _p, _p, _sz, _p]),
    "vb_ros2_stages": (_i, [_p, _i, _i, _p, _p, _p, _p, _p]),
    "vb_ros2_mixed_workspace_bytes": (_sz, [_i, _i, _i, _p]),
    "vb_ros2_step_mixed": (_i, [_p, _i, _i, _p, _p, _p, _p, _p, _i32, _p, _i, C.c_double, _p, _p, _p, _p, _p, _sz,
                                _p]),
    "vb_set_wait_limit": (_i, [C.c_longlong]),
    "vb_set_pipeline_wait_limit": (_i, [C.c_longlong]),
    "vb_set_factor_kernel": (_i, [_i]),
    "vb_chem_rhs": (_i, [_p, _i, _i, _p, _p, _p, _p, _p]),
    "vb_chem_jac": (_i, [_p, _i, _i, _p, _p, _p, _p, _p]),
    "vb_diffusion": (_i, [_i, _i, _i, _p, _p, _i32, _p, _p, _p, _p, _p]),
    "vb_bt_factor_bytes": (_sz, [_i, _i, _i]),
    "vb_bt_factor": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _p]),
    "vb_bt_solve": (_i, [_i, _i, _i, _p, _p, _p, _p]),
    "vb_bt_solve_T": (_i, [_i, _i, _i, _p, _p, _p, _p]),
    "vb_residual": (_i, [_p, _i, _i, _p, _p, _p, _p, _i32, _p, _p]),
    "vb_adjoint": (_i, [_p, _i, _i, _p, _p, _p, _p, _i32, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _sz, _p]),
    "vb_photo_tau": (_i, [_i, _i, _i, _p, _p, _p, _p, _p]),
    "vb_photo_flux": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "vb_photo_j": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _p]),
    "vb_photo_update": (_i, [_i, _i, _i, _i] + [_p] * 13 + [C.c_double, _p, _p]),
    "vb_rates": (_i, [_i, _i, _p, _p, _p, C.c_int32, _p, _p, _p]),
    "vb_atm_refresh": (_i, [_i, _i, _i] + [_p] * 12),
    "vb_loop_refresh": (_i, [_i, _i, _i, _p, C.c_int32] + [_p] * 12),
    "vb_conden_rates": (_i, [_i, _i, _i, _i, _i] + [_p] * 8),
    "vb_conden_relax": (_i, [_i, _i, _i] + [_p] * 8),
    "vb_profile": (_i, [_i]),
    "vb_profile_read": (_i, [_p, _p, _i]),
    "vb_fp64_probe": (_i, [_p, _i, _i, _i, _p]),
    "vb_ros2_step_static": (_i, [_p, _i, _i, _p, _p, _p, _p, _i32, _p, _p, _p, _p, _p]),
    "vb_adjoint_atm": (_i, [_i, _i, _i, _p, _p, _p, _i32, _p, _p, _p]),
    "vb_bt_mixed_bytes": (_sz, [_i, _i, _i]),
    "vb_bt_factor_mixed": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _p]),
    "vb_bt_solve_mixed": (_i, [_i, _i, _i, _p, _p, _p, _i, C.c_double, _p, _p, _p]),
    "vb_loop_body": (_i, [_i, _i, _i] + [_p] * 22),
    "vb_loop_condense": (_i, [_i, _i, _i, _i] + [_p] * 18),
    "vb_loop_converge": (_i, [_i, _i, _i] + [_p] * 13),
}

PROFILE_SITES = ["stage1_assembly", "factor", "back_sweep_1", "stage2_assembly", "forward_sweep_2",
                 "back_sweep_2"]

_LIB = None


class VulcanB200Error(RuntimeError):
    pass


def lib():
    """Load the library once (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise VulcanB200Error(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = h
    return _LIB


def check(code: int, what: str) -> None:
    if code != 0:
        msg = lib().vb_last_error().decode(errors="replace")
        raise VulcanB200Error(f"{what} failed (code {code}): {msg}")


def ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)
