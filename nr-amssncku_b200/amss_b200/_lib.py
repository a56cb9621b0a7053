"""Loads libamss_b200.so (the sm_100a kernels behind the C ABI of include/amss_b200.h).

There is no CPU fallback: if the library is missing, or no CUDA device is
usable, every call raises.
"""
import ctypes
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libamss_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_ROOT), "include", "amss_b200.h")

_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_lib = None


class AmssError(RuntimeError):
    """A library call failed; the message is the library's own."""


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AmssError(f"{LIB_PATH} is not built: run `make -C {PKG_ROOT}` (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    L.amss_last_error.restype = ctypes.c_char_p
    L.amss_version.restype = ctypes.c_char_p
    L.compute_rhs_bssn_.restype = ctypes.c_int
    L.compute_rhs_z4c_.restype = ctypes.c_int
    L.amss_compute_rhs_bssn_noalloc.restype = ctypes.c_int
    L.rungekutta4_rout_.restype = ctypes.c_int
    for name in ("sommerfeld_routbam_", "sommerfeld_rout_", "enforce_ga_", "lowerboundset_"):
        getattr(L, name).restype = None
    L.amss_engine_create.restype = ctypes.c_void_p
    L.amss_engine_create.argtypes = [ctypes.c_void_p]
    L.amss_engine_destroy.argtypes = [ctypes.c_void_p]
    L.amss_engine_destroy.restype = None
    L.amss_engine_add_block.argtypes = [ctypes.c_void_p, ctypes.c_int, _IP, _DP, _DP]
    L.amss_engine_commit.argtypes = [ctypes.c_void_p]
    L.amss_engine_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_engine_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_engine_state_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_longlong)]
    L.amss_engine_enforce.argtypes = [ctypes.c_void_p]
    L.amss_engine_step_level.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
    L.amss_engine_run_graph.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.amss_engine_sync.argtypes = [ctypes.c_void_p]
    L.amss_engine_stream.argtypes = [ctypes.c_void_p]
    L.amss_engine_stream.restype = ctypes.c_void_p
    L.amss_engine_set_grid.argtypes = [ctypes.c_void_p, _DP, ctypes.c_double]
    L.amss_engine_add_amr_block.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [_IP] * 6 + [ctypes.c_int]
    L.amss_engine_coarse_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
    L.amss_engine_run_coarse_graph.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.amss_engine_level_points.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.amss_engine_level_points.restype = ctypes.c_longlong
    L.amss_engine_launch_count.argtypes = [ctypes.c_void_p]
    L.amss_engine_launch_count.restype = ctypes.c_longlong
    L.amss_engine_constraint_norms.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_engine_set_punctures.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_engine_get_punctures.argtypes = [ctypes.c_void_p, _DP]
    L.amss_engine_interp_points.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _DP, ctypes.c_int, _IP, _DP,
                                            _DP, _IP]
    L.amss_engine_set_level_tiling.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.amss_engine_regrid_fill.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.amss_engine_set_time_level.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _DP]
    L.amss_engine_get_time_level.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _DP]
    L.amss_engine_level_clock.argtypes = [ctypes.c_void_p, ctypes.c_int, _IP]
    L.amss_engine_set_level_clock.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.amss_engine_get_level_tiling.argtypes = [ctypes.c_void_p, ctypes.c_int, _IP, _IP, _IP]
    L.get_lousto_nbhs_.restype = ctypes.c_int
    L.amss_lousto_vjp.restype = ctypes.c_int
    L.amss_lousto_vjp.argtypes = [_IP, _DP, _DP, _DP, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _DP]
    L.amss_adjoint_create.restype = ctypes.c_void_p
    L.amss_adjoint_create.argtypes = [_IP, _DP, ctypes.c_double, ctypes.c_double]
    L.amss_adjoint_destroy.restype = None
    L.amss_adjoint_destroy.argtypes = [ctypes.c_void_p]
    L.amss_adjoint_set_state.argtypes = [ctypes.c_void_p, _DP]
    L.amss_adjoint_get_state.argtypes = [ctypes.c_void_p, _DP]
    L.amss_adjoint_forward.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, _DP]
    L.amss_adjoint_backward.argtypes = [ctypes.c_void_p, _DP]
    L.amss_adjoint_stream.restype = ctypes.c_void_p
    L.amss_adjoint_stream.argtypes = [ctypes.c_void_p]
    L.amss_adjoint_launch_count.restype = ctypes.c_longlong
    L.amss_adjoint_launch_count.argtypes = [ctypes.c_void_p]
    L.amss_engine_set_rank.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.amss_engine_set_block_owner.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.amss_group_create.restype = ctypes.c_void_p
    L.amss_group_create.argtypes = [ctypes.c_int, ctypes.c_double]
    L.amss_group_destroy.restype = None
    L.amss_group_destroy.argtypes = [ctypes.c_void_p]
    L.amss_group_join.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.amss_group_barrier.argtypes = [ctypes.c_void_p]
    L.amss_nccl_unique_id.argtypes = [ctypes.c_char_p]
    L.amss_engine_set_nccl.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    L.amss_engine_constraint_sums.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_plan_create.restype = ctypes.c_void_p
    L.amss_plan_create.argtypes = [ctypes.c_void_p]
    L.amss_plan_commit.argtypes = [ctypes.c_void_p]
    L.amss_engine_xfer_count.argtypes = [ctypes.c_void_p]
    L.amss_engine_xfer_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    L.amss_engine_xfer_boxes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _IP, ctypes.c_int]
    L.amss_engine_xfer_peers.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    L.amss_engine_staging_block.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    L.amss_engine_psi4.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.amss_engine_get_psi4.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_engine_psi4_modes.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                         _DP, _DP]
    L.amss_engine_constraint_norms_first_patch.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP]
    L.amss_engine_set_level_occupancy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.amss_engine_get_level_occupancy.argtypes = [ctypes.c_void_p, ctypes.c_int, _IP]
    L.amss_engine_level_final_region.argtypes = [ctypes.c_void_p, ctypes.c_int, _IP, ctypes.POINTER(ctypes.c_longlong)]
    L.amss_engine_adm_integrals.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _DP]
    _lib = L
    return L


def last_error():
    return lib().amss_last_error().decode()


def check(rc, what):
    if rc < 0:
        raise AmssError(f"{what} failed ({rc}): {last_error()}")
    return rc


def header_functions():
    """Names of the functions include/amss_b200.h declares."""
    import re
    src = open(HEADER_PATH).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", src)) - {"if", "sizeof", "defined"})
