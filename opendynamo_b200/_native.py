"""ctypes binding of libopendynamo.so (the C ABI in include/opendynamo.h).

The shared library is built in-tree (``python -m opendynamo_b200.build``) and
there is no fallback: if it is missing, importing a solver raises.
"""

from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libopendynamo.so")

OD_FLUX = {"slau2": 0, "ausm+": 1, "rusanov": 2}
OD_F32, OD_F64 = 0, 1
OD_VISC_CONSTANT, OD_VISC_SUTHERLAND = 0, 1

ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "size mismatch", -4: "call out of order", -5: "I/O error",
          -6: "mesh exceeds the no-alloc scratch"}

# every symbol include/opendynamo.h declares
EXPORTS = (
    "od_default_params", "od_params_size", "od_abi_version", "od_create", "od_destroy", "od_state_bytes", "od_set_state", "od_get_state",
    "od_set_state_device", "od_get_state_device", "od_step", "od_rhs", "od_sync", "od_stream",
    "od_launches_per_step", "od_set_launch_shape", "od_set_pipeline_slabs", "od_set_timing", "od_timing", "od_last_error", "od_fr_tables",
    "od_rhs_noalloc", "od_make_initial_state", "od_state_save", "od_state_info", "od_state_load", "od_state_error", "od_run",
    "od_diagnostics",
    "od_ensemble_create", "od_ensemble_destroy", "od_ensemble_state_bytes", "od_ensemble_set_state",
    "od_ensemble_get_state", "od_ensemble_step", "od_ensemble_set_wait", "od_ensemble_set_shape", "od_ensemble_info",
    "od_ensemble_autotune", "od_ensemble_last_error", "od_ensemble_stream",
    "od_gemm_bf16", "od_mlp_wait_selftest",
    "od_mlp_create", "od_mlp_destroy", "od_mlp_last_error", "od_mlp_param_count", "od_mlp_set_params",
    "od_mlp_get_params", "od_mlp_forward", "od_mlp_gradients", "od_mlp_train_step", "od_mlp_set_scaling",
    "od_mlp_set_fused",
    "od_attach_closure", "od_project", "od_closure_features", "od_f32_to_bf16",
    "od_point_fields", "od_fields_save", "od_xdmf_text", "od_xdmf_convert",
    "od_get_state_async", "od_set_state_async", "od_create_slab", "od_slab_stage", "od_slab_halo_bytes", "od_slab_pack", "od_slab_unpack", "od_slabs_step",
)


class OdParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("flux", ctypes.c_int), ("y_wall", ctypes.c_int),
        ("u_real", ctypes.c_int), ("q_real", ctypes.c_int),
        ("rhs_real", ctypes.c_int), ("compute_real", ctypes.c_int),
        ("mixed", ctypes.c_int), ("fast_math", ctypes.c_int),
        ("mu", ctypes.c_double), ("forcing", ctypes.c_double),
        ("device", ctypes.c_int), ("ref_compat", ctypes.c_int),
        ("viscosity_model", ctypes.c_int), ("t_ref", ctypes.c_double), ("s_suth", ctypes.c_double),
    ]


class OdIcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("mach_bulk", ctypes.c_double), ("initial_condition", ctypes.c_int),
        ("perturbation_amplitude", ctypes.c_double), ("perturbation_modes", ctypes.c_int),
        ("perturbation_seed", ctypes.c_int),
    ]


OD_IC = {"channel": 0, "uniform": 1, "taylor-green": 2}


class OdRunOpts(ctypes.Structure):
    _fields_ = [
        ("initial_state", ctypes.c_char_p), ("n_steps", ctypes.c_longlong), ("dt", ctypes.c_double),
        ("save_freq", ctypes.c_longlong), ("checkpoint_freq", ctypes.c_longlong),
        ("compression", ctypes.c_char_p), ("output_dir", ctypes.c_char_p), ("prefix", ctypes.c_char_p),
        ("quiet", ctypes.c_int),
    ]


class OdRunResult(ctypes.Structure):
    _fields_ = [
        ("start_label", ctypes.c_ulonglong), ("final_label", ctypes.c_ulonglong),
        ("start_t", ctypes.c_double), ("final_t", ctypes.c_double),
        ("seconds", ctypes.c_double), ("ms_per_step", ctypes.c_double),
        ("files_written", ctypes.c_longlong), ("io_errors", ctypes.c_longlong),
        ("rho_min", ctypes.c_float), ("rho_max", ctypes.c_float),
        ("u_min", ctypes.c_float), ("u_max", ctypes.c_float),
    ]


class OdBox(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("flux", ctypes.c_int), ("y_wall", ctypes.c_int),
        ("mu", ctypes.c_double), ("forcing", ctypes.c_double), ("dt", ctypes.c_double),
    ]


class OdError(RuntimeError):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OdError(f"{LIB_PATH} is missing: build it with `python -m opendynamo_b200.build` "
                      "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, sz, ci, cd = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    P = ctypes.POINTER(OdParams)
    sig = {
        "od_default_params": (None, [P]),
        "od_params_size": (ctypes.c_size_t, []),
        "od_abi_version": (ci, []),
        "od_create": (ci, [P, ctypes.POINTER(vp)]),
        "od_destroy": (None, [vp]),
        "od_state_bytes": (sz, [vp]),
        "od_set_state": (ci, [vp, vp, sz]),
        "od_get_state": (ci, [vp, vp, sz]),
        "od_set_state_device": (ci, [vp, vp, sz]),
        "od_get_state_device": (ci, [vp, vp, sz]),
        "od_step": (ci, [vp, ci, cd]),
        "od_rhs": (ci, [vp, vp, sz]),
        "od_sync": (ci, [vp]),
        "od_stream": (vp, [vp]),
        "od_launches_per_step": (ci, [vp]),
        "od_set_launch_shape": (ci, [vp, ci, ci]),
        "od_set_pipeline_slabs": (ci, [vp, ci]),
        "od_set_timing": (ci, [vp, ci]),
        "od_timing": (ci, [vp, ctypes.POINTER(cd), ctypes.POINTER(cd), ctypes.POINTER(ctypes.c_longlong)]),
        "od_last_error": (ctypes.c_char_p, [vp]),
        "od_fr_tables": (ci, [vp]),
        "od_rhs_noalloc": (ci, [P, vp, vp, sz, vp]),
        "od_make_initial_state": (ci, [ctypes.POINTER(OdIcParams), vp, sz, ci]),
        "od_state_save": (ci, [ctypes.c_char_p, vp, ci, ci, ci, ci, ctypes.c_ulonglong, cd, cd, cd, cd,
                               ctypes.c_char_p]),
        "od_state_info": (ci, [ctypes.c_char_p, ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(ci),
                               ctypes.POINTER(ci), ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(cd),
                               ctypes.POINTER(cd), ctypes.POINTER(cd), ctypes.POINTER(cd), ctypes.c_char_p]),
        "od_state_load": (ci, [ctypes.c_char_p, vp, sz, ci, ci, ci, ci, ctypes.POINTER(ctypes.c_ulonglong),
                               ctypes.POINTER(cd)]),
        "od_state_error": (ctypes.c_char_p, []),
        "od_run": (ci, [P, ctypes.POINTER(OdRunOpts), ctypes.POINTER(OdRunResult), ctypes.c_char_p, sz]),
        "od_diagnostics": (ci, [vp, vp, vp, sz]),
        "od_ensemble_create": (ci, [ctypes.POINTER(OdBox), ci, ci, ci, ctypes.POINTER(vp)]),
        "od_ensemble_destroy": (None, [vp]),
        "od_ensemble_state_bytes": (sz, [vp, ci]),
        "od_ensemble_set_state": (ci, [vp, ci, vp, sz]),
        "od_ensemble_get_state": (ci, [vp, ci, vp, sz]),
        "od_ensemble_step": (ci, [vp, ci]),
        "od_ensemble_set_wait": (ci, [vp, ctypes.c_longlong, ci]),
        "od_mlp_wait_selftest": (ci, [ctypes.c_longlong, ci, ctypes.POINTER(ci), ctypes.POINTER(ci)]),
        "od_ensemble_set_shape": (ci, [vp, ci, ci, ci]),
        "od_ensemble_info": (ci, [vp, ctypes.POINTER(ci), ctypes.POINTER(ci), ctypes.POINTER(ci),
                                  ctypes.POINTER(ci)]),
        "od_ensemble_autotune": (ci, [vp, ci, ctypes.c_char_p, sz]),
        "od_ensemble_last_error": (ctypes.c_char_p, [vp]),
        "od_ensemble_stream": (vp, [vp]),
        "od_gemm_bf16": (ci, [ci, ci, ci, vp, vp, vp, vp, vp]),
        "od_mlp_create": (ci, [ci, ci, ctypes.POINTER(vp)]),
        "od_mlp_destroy": (None, [vp]),
        "od_mlp_last_error": (ctypes.c_char_p, [vp]),
        "od_mlp_param_count": (ctypes.c_longlong, [vp]),
        "od_mlp_set_params": (ci, [vp, vp]),
        "od_mlp_get_params": (ci, [vp, vp]),
        "od_mlp_forward": (ci, [vp, vp, ci, vp]),
        "od_mlp_gradients": (ci, [vp, vp, vp, vp, ci, ci, vp, ctypes.POINTER(cd)]),
        "od_mlp_train_step": (ci, [vp, vp, vp, vp, ci, ctypes.c_float, ctypes.POINTER(cd)]),
        "od_mlp_set_scaling": (ci, [vp, vp, vp, vp]),
        "od_mlp_set_fused": (ci, [vp, ci]),
        "od_attach_closure": (ci, [vp, vp]),
        "od_project": (ci, [vp, ci, ci, ci, ci, ci, vp, ci, vp]),
        "od_closure_features": (ci, [vp, ci, ci, ci, ci, cd, cd, cd, vp, vp, vp, vp]),
        "od_f32_to_bf16": (ci, [vp, vp, ctypes.c_longlong, vp]),
        "od_point_fields": (ci, [vp, ci, ci, ci, ci, vp, vp]),
        "od_fields_save": (ci, [ctypes.c_char_p, vp, ci, ctypes.POINTER(ctypes.c_char_p), ctypes.c_longlong,
                                ctypes.c_longlong, ctypes.c_longlong, ci, ctypes.c_char_p]),
        "od_xdmf_text": (ctypes.c_longlong, [ctypes.c_char_p, sz, ctypes.c_char_p, ci, ci, ci, cd, cd, cd,
                                             ctypes.c_ulonglong, cd]),
        "od_xdmf_convert": (ci, [ctypes.c_char_p, ctypes.c_char_p, sz, ctypes.c_char_p, sz, ctypes.c_char_p, ci]),
        "od_get_state_async": (ci, [vp, vp, sz, vp]),
        "od_set_state_async": (ci, [vp, vp, sz, vp]),
        "od_create_slab": (ci, [P, ci, ci, ctypes.POINTER(vp)]),
        "od_slab_stage": (ci, [vp, ci, ci, cd]),
        "od_slab_halo_bytes": (sz, [vp, ci, ci]),
        "od_slab_pack": (ci, [vp, ci, ci, ci, vp, vp]),
        "od_slab_unpack": (ci, [vp, ci, ci, ci, vp, vp]),
        "od_slabs_step": (ci, [ctypes.POINTER(vp), ci, ci, cd]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != 0:
        msg = ""
        if ctx:
            raw = lib().od_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise OdError(f"{what} failed ({ERRORS.get(rc, rc)}): {msg}")
