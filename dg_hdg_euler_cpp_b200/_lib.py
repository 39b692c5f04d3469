"""ctypes binding of the in-tree C ABI library lib/libdgh_gpu.so (include/dgh_gpu.h).

There is no CPU fallback: importing works anywhere, but load() raises when the library is
missing, and dgh_ctx_create fails without an sm_100 GPU.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libdgh_gpu.so"
BIN_PATH = PKG / "bin" / "dgh2d"
BIN1D_PATH = PKG / "bin" / "dgh1d"

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p


class dgh_config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("degree", ctypes.c_int), ("quadrature", ctypes.c_int),
        ("restart", ctypes.c_int), ("max_linear", ctypes.c_int), ("max_newton", ctypes.c_int), ("steps", ctypes.c_int),
        ("newton_steps", ctypes.c_int), ("warmup_updates", ctypes.c_int),
        ("cfl", ctypes.c_double), ("final_time", ctypes.c_double), ("safety", ctypes.c_double),
        ("nonlinear_tolerance", ctypes.c_double), ("linear_tolerance", ctypes.c_double),
        ("method", ctypes.c_int), ("integrator", ctypes.c_int), ("testcase", ctypes.c_int),
        ("precision", ctypes.c_int), ("check_update", ctypes.c_int), ("device", ctypes.c_int),
        ("dim", ctypes.c_int), ("autotune", ctypes.c_int),
        ("preconditioner", ctypes.c_int), ("condense32", ctypes.c_int), ("forcing", ctypes.c_int),
    ]


class dgh_update_stats(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_int), ("stage", ctypes.c_int), ("iteration", ctypes.c_int), ("krylov_iterations", ctypes.c_int),
        ("time", ctypes.c_double), ("stage_time", ctypes.c_double), ("dt", ctypes.c_double), ("cfl", ctypes.c_double),
        ("residual_physical_rms", ctypes.c_double), ("damping", ctypes.c_double),
        ("linear_relative_residual", ctypes.c_double), ("dg_linear_relative_residual", ctypes.c_double),
        ("iteration_s", ctypes.c_double),
    ]


class dgh_adjoint_stats(ctypes.Structure):
    _fields_ = [
        ("objective", ctypes.c_double), ("final_time", ctypes.c_double), ("steps", ctypes.c_int),
        ("checkpoints", ctypes.c_int), ("forward_newton", ctypes.c_int), ("adjoint_krylov", ctypes.c_int),
        ("recomputed_steps", ctypes.c_int),
    ]


class dgh_run_stats(ctypes.Structure):
    _fields_ = [
        ("final_time", ctypes.c_double), ("conservation_drift", ctypes.c_double), ("seconds", ctypes.c_double),
        ("max_linear_residual", ctypes.c_double), ("max_dg_linear_residual", ctypes.c_double),
        ("minimum_step", ctypes.c_double), ("maximum_step", ctypes.c_double),
        ("measured_newton_seconds", ctypes.c_double),
        ("steps", ctypes.c_int), ("newton_iterations", ctypes.c_int), ("krylov_iterations", ctypes.c_int),
        ("measured_updates", ctypes.c_int), ("updates_recorded", ctypes.c_int),
    ]


# name -> (restype, argtypes); every symbol declared in include/dgh_gpu.h
SIGNATURES = {
    "dgh_config_default": (None, [ctypes.POINTER(dgh_config)]),
    "dgh_ctx_create": (ctypes.c_int, [ctypes.POINTER(dgh_config), ctypes.POINTER(_VP)]),
    "dgh_ctx_destroy": (ctypes.c_int, [_VP]),
    "dgh_last_error": (ctypes.c_char_p, [_VP]),
    "dgh_sizes": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "dgh_get_config": (ctypes.c_int, [_VP, ctypes.POINTER(dgh_config)]),
    "dgh_stream": (_VP, [_VP]),
    "dgh_geometry": (ctypes.c_int, [_VP, _D]),
    "dgh_nodes": (ctypes.c_int, [_VP, _D, _D]),
    "dgh_sync": (ctypes.c_int, [_VP]),
    "dgh_device_bytes": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "dgh_launch_count": (ctypes.c_int64, [_VP]),
    "dgh_timing_enable": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dgh_timing_read": (ctypes.c_int, [_VP, ctypes.c_int, _D, ctypes.POINTER(ctypes.c_int64)]),
    "dgh_vec_alloc": (ctypes.c_int, [_VP, ctypes.c_int64, ctypes.POINTER(_D)]),
    "dgh_vec_free": (ctypes.c_int, [_VP, _D]),
    "dgh_upload": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int64]),
    "dgh_download": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int64]),
    "dgh_axpby": (ctypes.c_int, [_VP, ctypes.c_double, _VP, ctypes.c_double, _VP, _VP, ctypes.c_int64]),
    "dgh_initial": (ctypes.c_int, [_VP, _VP]),
    "dgh_freeze": (ctypes.c_int, [_VP, _VP, _D]),
    "dgh_set_stage": (ctypes.c_int, [_VP, _VP, ctypes.c_double]),
    "dgh_residual": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_admissible": (ctypes.c_int, [_VP, _VP, _I]),
    "dgh_trace": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_dual_norm": (ctypes.c_int, [_VP, _VP, _D]),
    "dgh_state_norm": (ctypes.c_int, [_VP, _VP, _D]),
    "dgh_integral": (ctypes.c_int, [_VP, _VP, _D]),
    "dgh_l2_error": (ctypes.c_int, [_VP, _VP, ctypes.c_double, _D]),
    "dgh_speeds": (ctypes.c_int, [_VP, _D]),
    "dgh_copy_speeds": (ctypes.c_int, [_VP, _VP]),
    "dgh_set_speeds": (ctypes.c_int, [_VP, _VP]),
    "dgh_mass_axpby": (ctypes.c_int, [_VP, ctypes.c_double, _VP, ctypes.c_double, _VP, _VP]),
    "dgh_rho2": (ctypes.c_int, [_VP, _VP, _D, _VP]),
    "dgh_dg_refresh": (ctypes.c_int, [_VP, _VP]),
    "dgh_dg_apply": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_dg_block": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "dgh_dg_apply_T": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_block_jacobi_refresh": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dgh_precond_apply": (ctypes.c_int, [_VP, ctypes.c_int, _VP, _VP]),
    "dgh_hdg_refresh_projected": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_hdg_rhs": (ctypes.c_int, [_VP, _VP]),
    "dgh_hdg_apply": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_hdg_block": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _D]),
    "dgh_hdg_recover": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_hdg_recovered_residual": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_hdg_retarget": (ctypes.c_int, [_VP, _VP]),
    "dgh_gmres": (ctypes.c_int, [_VP, ctypes.c_int, _VP, _VP, ctypes.c_int, ctypes.c_double, _I, _D]),
    "dgh_autotune_report": (ctypes.c_int, [_VP, _D]),
    "dgh_autotune_shapes": (ctypes.c_int, [_VP, _D]),
    "dgh_shape_set": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "dgh_gmres_graph_enable": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dgh_gmres_residual": (_VP, [_VP, ctypes.c_int]),
    "dgh_integrator_create": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(_VP)]),
    "dgh_integrator_destroy": (ctypes.c_int, [_VP]),
    "dgh_integrator_error": (ctypes.c_char_p, [_VP]),
    "dgh_advance": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(dgh_run_stats), ctypes.POINTER(dgh_update_stats), ctypes.c_int]),
    "dgh_stage_begin": (ctypes.c_int, [_VP, _VP, _D]),
    "dgh_newton_update": (ctypes.c_int, [_VP, ctypes.POINTER(dgh_update_stats)]),
    "dgh_newton_update_host": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(dgh_update_stats)]),
    "dgh_integrator_state": (_VP, [_VP]),
    "dgh_integrator_set_limits": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int]),
    "dgh_block_jacobi_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.POINTER(_VP)]),
    "dgh_block_jacobi_destroy": (ctypes.c_int, [_VP]),
    "dgh_block_jacobi_error": (ctypes.c_char_p, [_VP]),
    "dgh_block_jacobi_factor": (ctypes.c_int, [_VP, _VP]),
    "dgh_block_jacobi_apply": (ctypes.c_int, [_VP, _VP, _VP]),
    "dgh_block_jacobi_perm": (ctypes.c_int, [_VP, _I]),
    "dgh_dirk3_adjoint": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, ctypes.POINTER(dgh_adjoint_stats)]),
    "dgh_dirk3_replay": (ctypes.c_int, [_VP, _VP, _D]),
    "dgh_batch_create": (ctypes.c_int, [ctypes.POINTER(dgh_config), ctypes.c_int, ctypes.POINTER(_VP)]),
    "dgh_batch_destroy": (ctypes.c_int, [_VP]),
    "dgh_batch_error": (ctypes.c_char_p, [_VP, ctypes.c_int]),
    "dgh_batch_member": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(_VP), ctypes.POINTER(_VP)]),
    "dgh_batch_stage_begin": (ctypes.c_int, [_VP, _VP, _D, _I]),
    "dgh_batch_newton_update": (ctypes.c_int, [_VP, ctypes.POINTER(dgh_update_stats), _I]),
    "dgh_batch_download": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "dgh_batch_lockstep": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dgh_batch_lockstep_report": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "dgh_lockstep_create": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int, ctypes.POINTER(_VP)]),
    "dgh_lockstep_create_op": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP)]),
    "dgh_lockstep_destroy": (ctypes.c_int, [_VP]),
    "dgh_lockstep_error": (ctypes.c_char_p, []),
    "dgh_lockstep_begin": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dgh_lockstep_leave": (ctypes.c_int, [_VP, _VP]),
    "dgh_lockstep_report": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
    "dgh_residual_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            _VP, _VP, _VP, _VP, _VP, ctypes.c_char_p, ctypes.c_int]),
    "dgh_slab_rows": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _I]),
    "dgh_comm_local_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP)]),
    "dgh_comm_nccl_unique_id": (ctypes.c_int, [ctypes.POINTER(ctypes.c_ubyte)]),
    "dgh_comm_nccl_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(_VP)]),
    "dgh_comm_info": (ctypes.c_int, [_VP, _I]),
    "dgh_comm_fail": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "dgh_comm_set_timeout": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dgh_slab_halo_plan": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int64), _I]),
    "dgh_comm_destroy": (ctypes.c_int, [_VP]),
    "dgh_comm_error": (ctypes.c_char_p, []),
    "dgh_ctx_create_slab": (ctypes.c_int, [ctypes.POINTER(dgh_config), _VP, ctypes.POINTER(_VP)]),
    "dgh_slab_info": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64)]),
}

_lib = None


def build(verbose: bool = False) -> None:
    """Compile lib/libdgh_gpu.so and bin/dgh2d for sm_100a with the in-tree Makefile."""
    res = subprocess.run(["make", "-C", str(PKG / "csrc")], capture_output=True, text=True)
    if verbose or res.returncode != 0:
        print(res.stdout[-4000:], res.stderr[-4000:])
    if res.returncode != 0:
        raise RuntimeError("building libdgh_gpu.so failed")


def load(path: Path | None = None) -> ctypes.CDLL:
    """Load the CUDA library; raises when it has not been built (no fallback path exists).

    `path` selects another build of the same C ABI for the process; it must come before the
    first load."""
    global _lib
    if path is not None and _lib is not None and _lib._name != str(path):
        raise RuntimeError(f"{_lib._name} is already loaded in this process")
    if _lib is None:
        path = Path(path) if path is not None else LIB_PATH
        if not path.exists():
            raise RuntimeError(f"{path} is missing: build it with dg_hdg_euler_cpp_b200.build()")
        lib = ctypes.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
