"""ctypes binding of liblucky_droplets.so (the C ABI declared in include/ld.h).

The library is built in-tree by ``python -m lucky_droplets_b200.build``.  There is no CPU
fallback: if the library is missing or no CUDA device is present, every entry point raises.
"""
import ctypes
import pathlib

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "liblucky_droplets.so"

LD_OK = 0
LD_F32, LD_F64 = 0, 1
LD_INTERP = {"trilinear": 0, "tricubic": 1, "cosine": 2}
STATUS_NONFINITE = 1
STATUS_BLOWUP = 2
STATUS_PAIR_OVERFLOW = 4
STATUS_WAIT_TIMEOUT = 8

_c_p = ctypes.c_void_p
_c_i = ctypes.c_int
_c_i32 = ctypes.c_int32
_c_i64 = ctypes.c_int64
_c_d = ctypes.c_double
_c_dp = ctypes.POINTER(ctypes.c_double)


class FlowParams(ctypes.Structure):
    """ld_flow_params of include/ld.h."""
    _fields_ = [("dt", _c_d), ("nu", _c_d), ("f0", _c_d), ("kf_lo", _c_i32), ("kf_hi", _c_i32)]


class StepState(ctypes.Structure):
    """ld_step_state of include/ld.h."""
    _fields_ = [("uk", _c_p), ("ustar", _c_p), ("acc", _c_p), ("u4", _c_p), ("n", _c_i64), ("pos", _c_p),
                ("vel", _c_p), ("tau", _c_p), ("a1", _c_p), ("radius", _c_p), ("ids", _c_p), ("box", _c_p),
                ("method", _c_i32), ("g", _c_d), ("sort_every", _c_i32), ("order", _c_p), ("scratch", _c_p),
                ("pairs", _c_p), ("pair_cap", _c_i64), ("pair_count", _c_p), ("box_counts", _c_p),
                ("step", _c_i64)]


# name -> (restype, argtypes)
SIGNATURES = {
    "ld_version": (_c_i, []),
    "ld_last_error": (ctypes.c_char_p, []),
    "ld_plan_create": (_c_i, [ctypes.POINTER(_c_p), _c_i, _c_i]),
    "ld_plan_create_boxes": (_c_i, [ctypes.POINTER(_c_p), _c_i, _c_i, _c_i]),
    "ld_step": (_c_i, [_c_p, _c_p, ctypes.POINTER(StepState), ctypes.POINTER(FlowParams), _c_i32, _c_p]),
    "ld_ensemble_step": (_c_i, [_c_p, _c_p, ctypes.POINTER(StepState), ctypes.POINTER(FlowParams), _c_i32, _c_p]),
    "ld_plan_boxes": (_c_i, [_c_p, ctypes.POINTER(_c_i32)]),
    "ld_droplet_stage_boxes": (_c_i, [_c_p, _c_i, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_i, _c_d, _c_d, _c_p]),
    "ld_plan_destroy": (_c_i, [_c_p]),
    "ld_plan_dims": (_c_i, [_c_p, ctypes.POINTER(_c_i32), ctypes.POINTER(ctypes.c_size_t)]),
    "ld_rfft_mpi": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_p]),
    "ld_irfft_mpi": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_p]),
    "ld_irfft_mpi_noalloc": (_c_i, [_c_i, _c_p, _c_p, _c_i, _c_p]),
    "ld_irfft_cube": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_p]),
    "ld_rfft_cube": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_p]),
    "ld_spec_to_cube": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_p]),
    "ld_spec_from_cube": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_p]),
    "ld_spec_copy_region": (_c_i, [_c_p, _c_p, _c_p, _c_i, _c_i, _c_p]),
    "ld_shell_spectrum": (_c_i, [_c_p, _c_p, _c_p, _c_p]),
    "ld_velocity_rhs": (_c_i, [_c_p, _c_p, _c_p, _c_p, ctypes.POINTER(FlowParams), _c_d, _c_p]),
    "ld_rk2if_stage": (_c_i, [_c_p, _c_i, _c_p, _c_p, _c_p, _c_p, ctypes.POINTER(FlowParams), _c_p]),
    "ld_rk4_stage": (_c_i, [_c_p, _c_i, _c_p, _c_p, _c_p, _c_p, ctypes.POINTER(FlowParams), _c_p]),
    "ld_step_epilogue": (_c_i, [_c_p, _c_p, _c_p]),
    "ld_step_epilogue_plane0": (_c_i, [_c_p, _c_p, _c_p]),
    "ld_gather": (_c_i, [_c_p, _c_p, _c_i, _c_p, _c_i64, _c_i, _c_p, _c_p]),
    "ld_droplet_stage": (_c_i, [_c_p, _c_i, _c_p, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_i, _c_d, _c_d, _c_p]),
    "ld_profile": (_c_i, [_c_p, _c_i]),
    "ld_profile_read": (_c_i, [_c_p, ctypes.POINTER(_c_i32), ctypes.POINTER(_c_i64), _c_dp, _c_i,
                               ctypes.POINTER(_c_i32), _c_i]),
    "ld_kernel_name": (ctypes.c_char_p, [_c_i]),
    "ld_status": (_c_i, [_c_p, ctypes.POINTER(ctypes.c_uint32), _c_i, _c_p]),
    "ld_exact_sum": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_p]),
    "ld_mlp_sizes": (_c_i, [ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i32),
                            ctypes.POINTER(_c_i32)]),
    "ld_mlp_pack": (_c_i, [_c_p, _c_p, _c_p]),
    "ld_mlp_infer": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_p]),
    "ld_mlp_infer_ws": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_p]),
    "ld_mlp_infer_workspace_bytes": (_c_i64, [_c_i64]),
    "ld_phase_shift": (_c_i, [_c_p, _c_p, _c_p, _c_d, _c_d, _c_d, _c_p]),
    "ld_mlp_samples": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_d, _c_d, _c_d, _c_p, _c_p, _c_p, _c_p, _c_p]),
    "ld_interleave3": (_c_i, [_c_p, _c_p, _c_p, _c_p]),
    "ld_gather4": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_i, _c_p, _c_p]),
    "ld_mlp_partial_floats": (_c_i64, [_c_i64]),
    "ld_copy_async": (_c_i, [_c_p, _c_p, _c_i64, _c_p]),
    "ld_ref_workspace_doubles": (_c_i64, []),
    "ld_clip_zero": (_c_i, [_c_p, _c_p, _c_i64, _c_i, _c_p, _c_p]),
    "ld_axpy": (_c_i, [_c_p, _c_d, _c_p, _c_i64, _c_p]),
    "ld_waxpy": (_c_i, [_c_p, _c_p, _c_d, _c_p, _c_i64, _c_p]),
    "ld_n_products": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_p]),
    "ld_n_combine": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_p]),
    "ld_prhs_ref": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_d, _c_d, _c_d, _c_d, _c_d, _c_p, _c_p, _c_p]),
    "ld_extract_pos": (_c_i, [_c_p, _c_i64, _c_p, _c_p]),
    "ld_cell_weights": (_c_i, [_c_p, _c_i64, _c_i, _c_d, _c_p, _c_p, _c_p, _c_p]),
    "ld_cell_starts": (_c_i, [_c_p, _c_i64, _c_i64, _c_p, _c_p]),
    "ld_deposit_pull": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_i, _c_d, _c_p, _c_p]),
    "ld_slow_manifold": (_c_i, [_c_p, _c_p, _c_d, _c_d]),
    "ld_plan_autotune": (_c_i, [_c_p, _c_p, _c_p, _c_p]),
    "ld_plan_set_tuning": (_c_i, [_c_p, _c_p]),
    "ld_plan_set_wait_limit": (_c_i, [_c_p, ctypes.c_uint32, _c_i]),
    "ld_plan_prepare": (_c_i, [_c_p, ctypes.POINTER(FlowParams), _c_p]),
    "ld_shell_cross": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_p]),
    "ld_divergence_spec": (_c_i, [_c_p, _c_p, _c_p, _c_p]),
    "ld_droplet_predict": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_d, _c_p, _c_p]),
    "ld_droplet_update": (_c_i, [_c_p, _c_i, _c_p, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_d, _c_d, _c_p]),
    "ld_mlp_grad": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p]),
    "ld_mlp_adam": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_i64, ctypes.c_float, _c_p, _c_p]),
    "ld_mlp_train_epoch": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_i64, _c_p, _c_p, _c_p, _c_p, _c_i64, _c_d,
                                  _c_d, _c_i64, _c_p, _c_p, _c_p]),
    "ld_collider_create": (_c_i, [ctypes.POINTER(_c_p), _c_i64, _c_i32]),
    "ld_collider_create_boxes": (_c_i, [ctypes.POINTER(_c_p), _c_i64, _c_i32, _c_i32]),
    "ld_collide_boxes": (_c_i, [_c_p, _c_p, _c_p, _c_p, _c_i64, _c_d, _c_p, _c_i64, _c_p, _c_p, _c_p]),
    "ld_cell_order_boxes": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_d, _c_p, _c_p]),
    "ld_collider_destroy": (_c_i, [_c_p]),
    "ld_collide": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_d, _c_p, _c_i64, _c_p, _c_p]),
    "ld_collider_status": (_c_i, [_c_p, ctypes.POINTER(ctypes.c_uint32), _c_i, _c_p]),
    "ld_collider_trace": (_c_i, [_c_p, _c_p]),
    "ld_collider_sorted": (_c_i, [_c_p, ctypes.POINTER(_c_p), ctypes.POINTER(_c_p)]),
    "ld_radix_sort_u32": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_i, _c_p]),
    "ld_cell_order": (_c_i, [_c_p, _c_p, _c_i64, _c_d, _c_p, _c_p]),
    "ld_permute_rows": (_c_i, [_c_p, _c_p, _c_p, _c_i64, _c_i32, _c_p]),
}


class LDError(RuntimeError):
    """A negative status from the C ABI, with ld_last_error()'s message."""

    def __init__(self, code, msg):
        super().__init__(f"lucky_droplets error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load the library once and declare every signature; raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m lucky_droplets_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != LD_OK:
        raise LDError(rc, lib().ld_last_error().decode(errors="replace"))
    return rc


def ptr(t):
    """Raw device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)
