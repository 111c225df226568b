"""ctypes binding of libtrt_sweep.so (include/trt_sweep.h).

The library is the product: there is no Python or CPU implementation behind these names.  Loading
fails loudly when the shared library is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtrt_sweep.so")

TRT_OK = 0
TRT_ERR_ARG = -1
TRT_ERR_CUDA = -2
TRT_ERR_NOMEM = -3
TRT_ERR_BUDGET = -4
TRT_ERR_TIMEOUT = -5
TRT_ERR_STATE = -6
TRT_ERR_NODEV = -7
TRT_ERR_UNSUPPORTED = -8
TRT_ERR_SCRATCH = -9

TRT_PREC_FP64 = 0
TRT_PREC_FP32 = 1
TRT_CREATE_INPLACE = 0x10   # OR-ed into trt_create's precision: one in-place state buffer from the start

TRT_ROLL_STATE = 1
TRT_LAW_FLECK_CUMMINGS = 0   # material laws of the time loops (trt_tstep_set_law)
TRT_LAW_CONFIG = 1
TRT_MOMENTS = 2
TRT_RES_CALC = 4

# Field order of trt_moments_host (include/trt_sweep.h).
MOMENT_FIELDS = (
    "Hg_avg_xx", "Hg_avg_yy", "Hg_avg_xy", "Hg_edgV_xx", "Hg_edgV_xy", "Hg_edgH_yy", "Hg_edgH_xy",
    "Eg_avg", "Eg_edgV", "Eg_edgH", "Fxg_edgV", "Fyg_edgH",
    "fg_avg_xx", "fg_avg_yy", "fg_avg_xy", "fg_edgV_xx", "fg_edgV_xy", "fg_edgH_yy", "fg_edgH_xy",
    "Cg_L", "Cg_B", "Cg_R", "Cg_T",
    "Eg_in_L", "Eg_in_B", "Eg_in_R", "Eg_in_T", "Fg_in_L", "Fg_in_B", "Fg_in_R", "Fg_in_T",
    "E_avg", "E_edgV", "E_edgH", "Fx_edgV", "Fy_edgH",
    "E_in_L", "E_in_B", "E_in_R", "E_in_T", "F_in_L", "F_in_B", "F_in_R", "F_in_T",
    "Fyg_edgH_true", "Fy_edgH_true",
)


class MomentsHost(ctypes.Structure):
    _fields_ = [(n, ctypes.POINTER(ctypes.c_double)) for n in MOMENT_FIELDS]


def moment_shape(name, nx, ny, ng):
    """Fortran shape of a trt_moments_host field."""
    base = {"avg": (nx, ny), "edgV": (nx + 1, ny), "edgH": (nx, ny + 1)}
    if name.startswith("Cg_") or name.startswith("Eg_in_") or name.startswith("Fg_in_"):
        side = name[-1]
        return ((ny if side in "LR" else nx), ng)
    if name.startswith("E_in_") or name.startswith("F_in_"):
        return ((ny if name[-1] in "LR" else nx),)
    for key, shp in base.items():
        if key in name:
            grouped = "g_" in name or name.startswith("Hg") or name.startswith("fg") or name.startswith("Eg")
            return shp + (ng,) if grouped else shp
    raise KeyError(name)


class MlqdParams(ctypes.Structure):
    """trt_mlqd_params (include/trt_sweep.h)."""
    _fields_ = [("conv_lo", ctypes.c_double), ("conv_gr1", ctypes.c_double), ("conv_gr2", ctypes.c_double),
                ("maxit_mloqd", ctypes.c_int), ("maxit_gloqd", ctypes.c_int), ("chi", ctypes.c_double),
                ("line_src", ctypes.c_double), ("E_bound_low", ctypes.c_double), ("T_bound_low", ctypes.c_double),
                ("use_line_search", ctypes.c_int), ("use_safety_search", ctypes.c_int),
                ("kapE_dT_flag", ctypes.c_int), ("theta", ctypes.c_double), ("ho_form", ctypes.c_int)]


class MlqdStats(ctypes.Structure):
    """trt_mlqd_stats (include/trt_sweep.h)."""
    _fields_ = [("rt_its", ctypes.c_int), ("sweeps", ctypes.c_int), ("mgqd_its", ctypes.c_int),
                ("egp_its", ctypes.c_int), ("mgqd_nonconv", ctypes.c_int), ("egp_nonconv", ctypes.c_int),
                ("mgqd_krylov_max", ctypes.c_int), ("egp_krylov_max", ctypes.c_int),
                ("T_norm", ctypes.c_double), ("E_norm", ctypes.c_double), ("sweep_ms", ctypes.c_double),
                ("low_order_ms", ctypes.c_double), ("mgqd_solve_ms", ctypes.c_double), ("egp_ms", ctypes.c_double),
                ("mgqd_krylov_sum", ctypes.c_longlong), ("egp_krylov_sum", ctypes.c_longlong)]


# Exported symbols and their ctypes signatures.
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_i = ctypes.c_int
_d = ctypes.c_double
_P = ctypes.c_void_p
SIGNATURES = {
    "trt_transport_scb": (_i, [_i, _i, _i, _i] + [_D] * 6 + [_D] * 8 + [_d, _d, _i, _D, _I, _I, _i]),
    "trt_collapse_intensities": (_i, [_i, _i, _i, _i, _i, _D, _D, _D, _D, _D, _D, _d] + [_D] * 17),
    "trt_fg_calc": (_i, [_i, _i, _i] + [_D] * 7 + [_D] * 10 + [_d, _i]),
    "trt_cg_calc": (_i, [_i, _i, _i, _i] + [_D] * 4 + [_D] * 5 + [_d, _I, _i]),
    "trt_mgqd_in_calc": (_i, [_i, _i, _i, _i] + [_D] * 8 + [_D] * 5 + [_d, _d, _I, _i]),
    "trt_gqd_in_calc": (_i, [_i, _i, _i] + [_D] * 16),
    "trt_rt_bc_update": (_i, [_i, _i, _i, _i, _I, _d, _d, _d, _d, _d, _D, _D, _D, _D, _D]),
    "trt_bg_planck": (_d, [_d, _d, _d, _d]),
    "trt_create": (_P, [_i, _i, _i, _i, _D, _D, _D, _D, _D, _i, ctypes.c_size_t, _I]),
    "trt_destroy": (None, [_P]),
    "trt_required_bytes": (ctypes.c_size_t, [_i, _i, _i, _i, _i]),
    "trt_set_tiling": (_i, [_P, _i, _i, _i, _i]),
    "trt_get_tiling": (_i, [_P, _I, _I, _I, _I, _I]),
    "trt_set_material": (_i, [_P, _D, _D, _d, _d, _d]),
    "trt_set_material_device": (_i, [_P, _P, _P, _d, _d, _d]),
    "trt_set_material_async": (_i, [_P, _D, _D, _d, _d, _d]),
    "trt_moments_async": (_i, [_P, ctypes.POINTER(MomentsHost)]),
    "trt_set_source_full": (_i, [_P, _D]),
    "trt_set_boundary": (_i, [_P, _D, _D, _I]),
    "trt_bc_update": (_i, [_P, _I, _d, _d, _d, _d, _d, _D]),
    "trt_init_state": (_i, [_P, _d, _d, _d, _d, _d, _d, _D]),
    "trt_put_state": (_i, [_P, _D]),
    "trt_get_state": (_i, [_P, _D]),
    "trt_sweep": (_i, [_P, ctypes.c_uint]),
    "trt_sync": (_i, [_P]),
    "trt_moments": (_i, [_P, ctypes.POINTER(MomentsHost)]),
    "trt_get_angular": (_i, [_P, _D, _D, _D, _D, _D]),
    "trt_get_residual": (_i, [_P, _D, _I, _I]),
    "trt_snapshot_angular": (_i, [_P, _P]),
    "trt_snapshot_output": (_i, [_P, ctypes.c_char_p, _P]),
    "trt_stream": (_P, [_P]),
    "trt_set_wait_limit": (_i, [_P, ctypes.c_uint]),
    "trt_set_wait_limit_zero": (_i, [_P]),
    "trt_device_output": (_P, [_P, ctypes.c_char_p]),
    "trt_set_register_mode": (_i, [_P, _i]),
    "trt_set_bands": (_i, [_P, _i]),
    "trt_batch_set_persistent": (_i, [_P, _i]),
    "trt_set_inplace": (_i, [_P, _i]),
    "trt_state_bytes": (ctypes.c_size_t, [_P]),
    "trt_bind_state": (_i, [_P, ctypes.c_void_p, ctypes.c_size_t]),
    "trt_state_written": (_i, [_P]),
    "trt_snapshot_angular_groups": (_i, [_P, _i, _i, ctypes.c_void_p]),
    "trt_get_bands": (_i, [_P]),
    "trt_get_register_mode": (_i, [_P]),
    "trt_autotune": (_i, [_P, _I, _I, _I, ctypes.POINTER(ctypes.c_float)]),
    "trt_batch_create": (_P, [ctypes.POINTER(_P), _i, _I]),
    "trt_batch_destroy": (None, [_P]),
    "trt_batch_sweep": (_i, [_P, ctypes.c_uint]),
    "trt_batch_sync": (_i, [_P]),
    "trt_batch_tstep": (_i, [_P, _I, _D, _D]),
    "trt_tstep_setup": (_i, [_P, _D, _D, _D, _D, _d, _d, _d, _d, _I, _D, _i, _d, _i]),
    "trt_tstep": (_i, [_P, _I, _D, _D]),
    "trt_tstep_set_law": (_i, [_P, _i]),
    "trt_tstep_begin": (_i, [_P]),
    "trt_tstep_sweep": (_i, [_P, _i]),
    "trt_tstep_partials": (_i, [_P, ctypes.c_void_p]),
    "trt_tstep_finish": (_i, [_P, ctypes.c_void_p, _i, _I, _D, _D]),
    "trt_get_temperature": (_i, [_P, _D]),
    "trt_put_temperature": (_i, [_P, _D]),
    "trt_strerror": (ctypes.c_char_p, [_i]),
    "trt_kernel_launches": (ctypes.c_ulonglong, []),
    "trt_transport_residual_noalloc": (_i, [_i, _i, _i, _i] + [_P] * 11 + [_d, _d, _P, _P, _P, _P]),
    "trt_old_mgqd_coefs": (_i, [_i, _i, _i] + [_D] * 17 + [_d, _d, _d] + [_D] * 5 + [_i]),
    "trt_mloqd_fv": (_i, [_i, _i, _i] + [_D] * 29 + [_d, _d, _d, _i, _i] + [_D] * 10 + [_I, _d, _d, _d]),
    "trt_mgqd_set_tolerance": (_i, [_d, _i]),
    "trt_mgqd_set_graphs": (_i, [_i]),
    "trt_mgqd_set_fused_levels": (_i, [_i]),
    "trt_mgqd_set_smem_vcycle": (_i, [_i]),
    "trt_collapse_mg_ef": (_i, [_i, _i, _i] + [_D] * 5 + [_i] + [_D] * 5),
    "trt_cbar_calc": (_i, [_i, _i, _i] + [_D] * 15),
    "trt_old_grey_coefs": (_i, [_i, _i, _i, _d, _d, _d, _d] + [_D] * 8),
    "trt_grey_coefs": (_i, [_i, _i, _i] + [_D] * 14 + [_d, _d, _d] + [_D] * 4 + [_D] * 15 + [_d]),
    "trt_egp_fv_newt": (_i, [_i, _i] + [_D] * 9 + [_I, _D, _D, _D, _D, _d, _d] + [_D] * 3 + [_D] * 12 + [_D] * 14
                        + [_D] * 2 + [_d] * 9 + [_i] * 6 + [_I, _d, _d]),
    "trt_mgqd_last_stats": (_i, [_D, _I, _D]),
    "trt_pod_calc": (_i, [_D, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, _D, _D, _D,
                          _D]),
    "trt_pod_calc_device": (_i, [_P, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
                                 _P, _P, _P, _P, _P]),
    "trt_pod_reconstruct": (_i, [_D, _D, _D, _D, _D, _I, _i, _i, _i, _i, _i]),
    "trt_pod_reconstruct_device": (_i, [_P, _P, _P, _P, _P, _P, _P, _i, _i, _i, _i, _P]),
    "trt_dmd_reconstruct": (_i, [_D, _D, _D, _D, _D, _I, _i, _i, _i, _d]),
    "trt_fmap": (_i, [_D, _D, _D, _D, _I, _I, _i, _i, _i, _i]),
    "trt_linear_interpolation": (_i, [_D, _D, _d, _d, _d, _i]),
    "trt_gridmap_gen": (_i, [_i, _D, _D, _i, _i, _D]),
    "trt_map_grids": (_i, [_I, _D, _D, _i, _i, _i, _I]),
    "trt_generate_grids_t": (_i, [_d, _d, _d, _d, _i, _i, _D, _D, _I]),
    "trt_gridmap_gen_bnd": (_i, [_i, _D, _d, _i, _D]),
    "trt_rrank_calc": (_i, [_D, _d, _i, _I]),
    "trt_pod_reconstruct_fg_device": (_i, [_P] * 30 + [_I] * 6 + [_i] * 10 + [_P] * 6 + [_D] * 2 + [_P] * 6 + [_I, _P]),
    "trt_pod_reconstruct_bcg_device": (_i, [_P] * 8 + [_I] + [_i] * 10 + [_P] * 2 + [_D] * 2 + [_P] * 2 + [_I, _P]),
    "trt_pod_reconstruct_fg": (_i, [_D] * 30 + [_I] * 6 + [_i] * 10 + [_D] * 8 + [_I] * 7),
    "trt_pod_reconstruct_bcg": (_i, [_D] * 8 + [_I] + [_i] * 10 + [_D] * 4 + [_I] * 3),
    "trt_dmd_reconstruct_fg": (_i, [_D] * 30 + [_I] * 6 + [_i] * 6 + [_d, _i] + [_D] * 6 + [_I] * 6),
    "trt_dmd_reconstruct_bcg": (_i, [_D] * 8 + [_I] + [_i] * 6 + [_d, _i] + [_D] * 2 + [_I] * 2),
    "trt_generate_grids_xy": (_i, [_D, _D, _D, _D, _d, _d, _d, _d, _i, _i, _i, _i] + [_D] * 8 + [_I] * 8),
    "trt_collect_lr_bnd": (_i, [_D, _D, _i, _i, _i]),
    "trt_collect_bt_bnd": (_i, [_D, _D, _i, _i, _i]),
    "trt_collect_crn_bnd": (_i, [_D, _D, _i, _i, _i]),
    "trt_extnd_bt_bnd": (_i, [_D, _D, _i, _i, _i]),
    "trt_extnd_lr_bnd": (_i, [_D, _D, _i, _i, _i]),
    "trt_avg_apnd_bnd": (_i, [_D, _D, _D, _D, _D, _i, _i, _i]),
    "trt_dmd_calc": (_i, [_D, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, _i, _d, _d,
                          ctypes.POINTER(ctypes.c_longlong)] + [_D] * 8),
    "trt_mlqd_setup": (_i, [_P, _d, ctypes.POINTER(MlqdParams)]),
    "trt_mlqd_setup_range": (_i, [_P, _d, ctypes.POINTER(MlqdParams), _i, _i, _D]),
    "trt_mlqd_step": (_i, [_P, ctypes.POINTER(MlqdStats)]),
    "trt_mlqd_exchange_size": (ctypes.c_longlong, [_P]),
    "trt_mlqd_step_begin": (_i, [_P, _P]),
    "trt_mlqd_step_begin_finish": (_i, [_P, _P]),
    "trt_mlqd_outer_begin": (_i, [_P, _i, _P]),
    "trt_mlqd_outer_begin_finish": (_i, [_P, _P]),
    "trt_mlqd_mgqd_local": (_i, [_P, _P]),
    "trt_mlqd_mgqd_finish": (_i, [_P, _i, _P, _I]),
    "trt_mlqd_outer_end": (_i, [_P, _i, _I]),
    "trt_mlqd_step_end": (_i, [_P, ctypes.POINTER(MlqdStats)]),
    "trt_mlqd_counts": (_i, [_P, _I, _i, _I, _i, _I, _I]),
    "trt_mlqd_get": (_i, [_P, ctypes.c_char_p, _D, ctypes.c_longlong]),
    "trt_mlqd_put": (_i, [_P, ctypes.c_char_p, _P, ctypes.c_longlong, _i]),
}

_lib = None


class TrtError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        msg = lib().trt_strerror(code).decode() if _lib is not None else str(code)
        super().__init__(f"{where}: {msg} (code {code})")


def lib():
    """Load libtrt_sweep.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m` the package build "
                              "(__graft_entry__.build()) -- there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code, where):
    if code != TRT_OK:
        raise TrtError(code, where)


def dptr(a):
    """double* of a contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous), "need a contiguous float64 array"
    return a.ctypes.data_as(_D)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(_I)
