"""ctypes binding of librbffd_sm100.so (the C ABI in include/rbffd_sm100.h).

Loading fails loudly when the shared library has not been built: there is no
CPU fallback for any product entry point.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librbffd_sm100.so")

c_int, c_uint, c_double, c_size_t, c_void_p, c_char_p = (ctypes.c_int, ctypes.c_uint, ctypes.c_double, ctypes.c_size_t,
                                                          ctypes.c_void_p, ctypes.c_char_p)
c_uint64 = ctypes.c_uint64
P = ctypes.POINTER
dp = P(c_double)
ip = P(c_int)


class WeightParams(ctypes.Structure):
    _fields_ = [("der_types", c_uint), ("dim", c_int), ("poly_deg", c_int), ("hv_k", c_int), ("hv_gamma", c_double),
                ("hv_nodes", c_double)]


class PdeParams(ctypes.Structure):
    _fields_ = [("rhs_kind", c_int), ("ntracers", c_int), ("dtype", c_int), ("use_hv", c_int),
                ("sphere_radius", c_double), ("alpha", c_double), ("u0", c_double), ("kappa", c_double),
                ("cu", dp), ("cv", dp)]


class Request(ctypes.Structure):
    _fields_ = [("grid", c_void_p), ("pde", PdeParams), ("u0", dp), ("dt", c_double), ("nsteps", c_int),
                ("out", dp)]


class EigOutput(ctypes.Structure):
    _fields_ = [(k, c_double) for k in ("max_pos_eig", "min_pos_eig", "max_neg_eig", "min_neg_eig")] + \
               [(k, c_int) for k in ("nb_positive", "nb_negative", "nb_zero")]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_longlong) for k in ("submitted", "completed", "failed", "cancelled", "pending", "active",
                                                 "max_active_seen", "ticks", "launches", "slots_reused")] + \
               [(k, c_double) for k in ("node_updates", "gpu_busy_s", "stage_bytes", "budget_bytes", "held_bytes")]


# name -> (restype, argtypes)
PROTOTYPES = {
    "rbffd_version": (c_char_p, []),
    "rbffd_status_string": (c_char_p, [c_int]),
    "rbffd_device_count": (c_int, [ip]),
    "rbffd_ctx_create": (c_int, [c_int, P(c_void_p)]),
    "rbffd_ctx_destroy": (c_int, [c_void_p]),
    "rbffd_ctx_last_error": (c_char_p, [c_void_p]),
    "rbffd_ctx_synchronize": (c_int, [c_void_p]),
    "rbffd_ctx_mem_info": (c_int, [c_void_p, P(c_size_t), P(c_size_t), P(c_size_t)]),
    "rbffd_ctx_stream": (c_int, [c_void_p, P(c_void_p)]),
    "rbffd_ctx_set_arithmetic": (c_int, [c_void_p, c_int]),
    "rbffd_ctx_get_arithmetic": (c_int, [c_void_p, ip]),
    "rbffd_nodes_fibonacci": (c_int, [c_int, c_uint64, dp]),
    "rbffd_stencils_knn": (c_int, [dp, c_int, c_int, ip, ip, c_int]),
    "rbffd_stencils_generate": (c_int, [dp, c_int, c_int, c_int, c_double, ip, ip, ip, c_int]),
    "rbffd_variable_epsilon": (c_int, [c_int, dp, c_int, ip, ip, c_double, dp]),
    "rbffd_stencils_generate_gpu": (c_int, [c_void_p, dp, c_int, c_int, c_int, c_double, ip, ip, ip]),
    "rbffd_stencils_knn_gpu": (c_int, [c_void_p, dp, c_int, c_int, ip, ip]),
    "rbffd_exact_cosine_bell": (c_int, [c_int, dp, c_double, dp]),
    "rbffd_exact_sph_heat": (c_int, [c_int, dp, c_int, dp, c_double, c_double, dp]),
    "rbffd_grid_create": (c_int, [c_void_p, c_int, dp, c_int, ip, ip, P(c_void_p)]),
    "rbffd_grid_create_ordered": (c_int, [c_void_p, c_int, dp, c_int, ip, ip, c_int, P(c_void_p)]),
    "rbffd_node_order": (c_int, [c_int, dp, c_int, ip, ip, c_int, ip]),
    "rbffd_stencils_hash": (c_int, [dp, c_int, c_int, c_int, c_int, c_int, dp, c_double, ip, ip, ip]),
    "rbffd_vortex_rollup_coefficients": (c_int, [c_int, dp, dp]),
    "rbffd_exact_vortex_rollup": (c_int, [c_int, dp, c_double, dp]),
    "rbffd_sol_norms": (c_int, [dp, dp, c_int, dp]),
    "rbffd_grid_destroy": (c_int, [c_void_p]),
    "rbffd_grid_nbytes": (c_int, [c_void_p, P(c_size_t)]),
    "rbffd_weights_compute": (c_int, [c_void_p, P(WeightParams), dp, c_double, ip]),
    "rbffd_weights_assemble": (c_int, [c_void_p, P(WeightParams), dp, c_double, ip, ip, c_int, dp]),
    "rbffd_weights_set_elimination": (c_int, [c_void_p, c_int]),
    "rbffd_weights_get_elimination": (c_int, [c_void_p, ip]),
    "rbffd_weights_set": (c_int, [c_void_p, c_uint, dp]),
    "rbffd_weights_get": (c_int, [c_void_p, c_uint, dp]),
    "rbffd_weights_file_write": (c_int, [c_char_p, c_int, c_int, c_int, ip, ip, dp]),
    "rbffd_weights_file_read": (c_int, [c_char_p, c_int, c_int, c_int, ip, ip, dp]),
    "rbffd_eig_classify": (c_int, [dp, c_int, c_double, c_void_p, dp]),
    "rbffd_eigenvalues": (c_int, [c_void_p, c_uint, c_int, dp, dp, c_void_p, dp]),
    "rbffd_eigen_rightmost": (c_int, [c_void_p, c_uint, c_int, c_int, c_int, c_double, c_int, ctypes.c_ulonglong, dp,
                                      dp, dp, ip, ip, ip]),
    "rbffd_hessenberg_eigenvalues": (c_int, [c_int, dp, dp, dp]),
    "rbffd_apply": (c_int, [c_void_p, c_uint, c_int, c_uint, c_uint, dp, dp]),
    "rbffd_apply_dev": (c_int, [c_void_p, c_uint, c_int, c_int, c_void_p, c_void_p]),
    "rbffd_batched_gesv_dev": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "rbffd_pde_create": (c_int, [c_void_p, P(PdeParams), P(c_void_p)]),
    "rbffd_pde_destroy": (c_int, [c_void_p]),
    "rbffd_pde_set_state": (c_int, [c_void_p, dp]),
    "rbffd_pde_get_state": (c_int, [c_void_p, dp]),
    "rbffd_pde_set_time": (c_int, [c_void_p, c_double]),
    "rbffd_pde_get_time": (c_int, [c_void_p, dp]),
    "rbffd_pde_advance": (c_int, [c_void_p, c_int, c_double, c_int, c_int]),
    "rbffd_pde_set_shape": (c_int, [c_void_p, c_int, c_int]),
    "rbffd_pde_set_arithmetic": (c_int, [c_void_p, c_int]),
    "rbffd_pde_get_arithmetic": (c_int, [c_void_p, ip]),
    "rbffd_pde_set_fused_operator": (c_int, [c_void_p, c_int]),
    "rbffd_pde_set_compensated_state": (c_int, [c_void_p, c_int]),
    "rbffd_pde_set_tiled_shape": (c_int, [c_void_p, c_int, c_int, c_int]),
    "rbffd_pde_get_tiling": (c_int, [c_void_p, ip]),
    "rbffd_pde_get_tile_flags": (c_int, [c_void_p, ip]),
    "rbffd_heat_rk4_noalloc": (c_int, [c_void_p, c_int, c_double, c_double, c_int, c_void_p]),
    "rbffd_pde_get_shape": (c_int, [c_void_p, ip, ip]),
    "rbffd_server_start": (c_int, [c_void_p, c_double, c_int, P(c_void_p)]),
    "rbffd_server_submit": (c_int, [c_void_p, P(Request), P(c_uint64)]),
    "rbffd_server_poll": (c_int, [c_void_p, c_uint64, ip, ip, dp, dp]),
    "rbffd_server_wait": (c_int, [c_void_p, c_uint64, c_double]),
    "rbffd_server_wait_idle": (c_int, [c_void_p, c_double]),
    "rbffd_server_cancel": (c_int, [c_void_p, c_uint64]),
    "rbffd_server_get_stats": (c_int, [c_void_p, P(ServerStats)]),
    "rbffd_server_pause": (c_int, [c_void_p, c_int]),
    "rbffd_server_set_admission_order": (c_int, [c_void_p, c_int]),
    "rbffd_server_inject_admission_failures": (c_int, [c_void_p, c_int]),
    "rbffd_server_stop": (c_int, [c_void_p]),
}

_LIB = None


def load():
    """Load the built library; raises if it is missing (no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("librbffd_sm100.so is not built (run __graft_entry__.build() or "
                              "python rbffd_gpu_b200/build.py): " + LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB
