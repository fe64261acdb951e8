"""ctypes binding of libmstm_b200.so (the C ABI in include/mstm_b200.h).

The library is built in-tree (mstm_b200/libmstm_b200.so).  There is no CPU
fallback: if the library is missing or cannot be loaded, ``lib()`` raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmstm_b200.so")
_lib = None

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
P = ctypes.POINTER

# Every symbol include/mstm_b200.h declares, with (restype, argtypes).
SIGNATURES = {
    "mstmg_default_opts": (None, [c_void_p]),
    "mstmg_ctx_create": (c_int, [P(c_void_p), c_int, c_void_p, c_void_p, c_void_p, c_double, c_void_p]),
    "mstmg_ctx_destroy": (None, [c_void_p]),
    "mstmg_ctx_set_positions": (c_int, [c_void_p, c_void_p]),
    "mstmg_neqns": (c_int, [c_void_p]),
    "mstmg_npairs": (c_int, [c_void_p]),
    "mstmg_sphere_orders": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mstmg_mie_coefficients": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mstmg_vol_radius": (c_double, [c_void_p]),
    "mstmg_host_spheres": (c_int, [c_void_p, c_void_p]),
    "mstmg_host_mie_coefficients": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mstmg_interaction": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "mstmg_bicg": (c_int, [c_void_p, c_int, c_double, c_void_p, c_void_p, c_int, P(c_int), P(c_double)]),
    "mstmg_planewave": (c_int, [c_void_p, c_double, c_double, c_int, c_void_p]),
    "mstmg_ensemble_create": (c_int, [P(c_void_p), c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_double, c_void_p]),
    "mstmg_ensemble_fixed_orientation": (c_int, [c_void_p, c_double, c_double, c_int, c_double, c_int, c_void_p, c_void_p, c_void_p,
                                                 c_void_p, c_void_p]),
    "mstmg_fixed_orientation": (c_int, [c_void_p, c_double, c_double, c_int, c_double, c_int, c_void_p, c_void_p, c_void_p,
                                        P(c_double), P(c_int)]),
    "mstmg_scattering": (c_int, [c_void_p, c_void_p, c_double, c_int, c_int, c_void_p, P(c_double), P(c_int), c_void_p,
                                 c_int]),
    "mstmg_selftest_bounded_wait": (c_int, [c_int, c_int, P(c_int)]),
    "mstmg_interaction_ex": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int]),
    "mstmg_translation_pass": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "mstmg_gsf_coefficients": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "mstmg_scattering_plane": (c_int, [c_void_p, c_int, c_void_p, c_int, c_int, c_double, c_double, c_double, c_int, c_void_p]),
    "mstmg_t_matrix_order": (c_int, [c_void_p, c_double, c_int, P(c_int)]),
    "mstmg_tmatrix": (c_int, [c_void_p, c_int, c_double, c_double, c_int, c_void_p, c_void_p, c_void_p, P(c_int), P(c_int),
                              P(c_double)]),
    "mstmg_tmatrix_qext_qsca": (c_int, [c_void_p, c_int, c_void_p, P(c_double), P(c_double)]),
    "mstmg_ranorient_scattering": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "mstmg_fft_setup": (c_int, [c_void_p, c_double, c_double, c_int, c_int, c_void_p, P(c_double), P(c_int), P(c_int)]),
    "mstmg_fixed_orientation_guess": (c_int, [c_void_p, c_double, c_double, c_int, c_double, c_int, c_void_p, c_double, c_void_p,
                                              c_void_p, c_void_p, c_void_p, c_void_p, P(c_double), P(c_int)]),
    "mstmg_nn_gemm": (c_int, [c_int, c_int, c_int, c_void_p, c_int, c_int, c_void_p, c_int, c_int, c_int, c_void_p, c_int, c_int,
                              c_void_p]),
    "mstmg_nn_bias_act": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "mstmg_nn_act_back": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "mstmg_nn_colsum": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_edge_concat": (c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_edge_concat_back": (c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_scatter_add": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_gather": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "mstmg_nn_mse": (c_int, [ctypes.c_longlong, c_void_p, c_void_p, c_void_p, ctypes.c_float, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_adam": (c_int, [ctypes.c_longlong, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_float, ctypes.c_float,
                              ctypes.c_float, ctypes.c_float, c_int, c_void_p]),
    "mstmg_nn_to_bf16": (c_int, [ctypes.c_longlong, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_axpy": (c_int, [ctypes.c_longlong, ctypes.c_float, c_void_p, c_void_p, c_void_p]),
    "mstmg_nn_knn": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mstmg_last_stats": (c_int, [c_void_p, c_void_p, P(c_int), P(c_int), P(c_int)]),
    "mstmg_operator_bytes": (c_int, [c_void_p, c_int, P(c_double), P(c_double)]),
    "mstmg_time_translation": (c_int, [c_void_p, c_int, c_int, c_int, P(c_double)]),
    "mstmg_set_stream": (c_int, [c_void_p, c_void_p]),
    "mstmg_set_timing": (c_int, [c_void_p, c_int]),
    "mstmg_kernel_time": (c_int, [c_void_p, P(c_double), P(c_int), P(c_double), P(c_int)]),
    "mstmg_kernel_time_tc": (c_int, [c_void_p, P(c_double), P(c_int)]),
    "mstmg_last_host_syncs": (c_int, [c_void_p]),
    "mstmg_set_pair_shard": (c_int, [c_void_p, c_int, c_int]),
    "mstmg_fixed_orientation_rhs": (c_int, [c_void_p, c_double, c_double, c_int, c_void_p]),
    "mstmg_efficiencies": (c_int, [c_void_p, c_double, c_double, c_int, c_void_p, c_void_p, c_void_p]),
    "mstmg_kernel_launches": (ctypes.c_longlong, []),
    "mstmg_planewave_noalloc": (c_int, [c_int, c_int, c_void_p, c_double, c_double, c_int, c_void_p, c_void_p]),
    "mstmg_last_error": (ctypes.c_char_p, []),
}


class MstmgOpts(ctypes.Structure):
    _fields_ = [("precision", c_int), ("device", c_int), ("medium_re", c_double), ("medium_im", c_double),
                ("translation_switch_order", c_int), ("inner_eps", c_double), ("max_outer", c_int),
                ("generic_kernel", c_int), ("tile_ctas_per_sm", c_int), ("fp32_chunk", c_int),
                ("mixed_solver", c_int), ("gmres_restart", c_int), ("tile_pairs", c_int), ("tensor_core", c_int)]


class MstmgError(RuntimeError):
    def __init__(self, code, where):
        msg = lib().mstmg_last_error().decode(errors="replace")
        super().__init__("%s failed with status %d: %s" % (where, code, msg))
        self.code = code


def lib():
    """Load the CUDA library; raises if it was not built (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libmstm_b200.so is not built; run `python -m mstm_b200.build` "
                               "(the CUDA extension is required, there is no CPU path)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code, where):
    if code < 0:
        raise MstmgError(code, where)
    return code
