"""ctypes binding of libfeb200.so (the C ABI declared in include/feb200.h).

The library is loaded from this package directory (built in-tree by ``python -m comech_b200.build``).
There is no fallback: if the library or a CUDA device is missing, every entry point raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfeb200.so")

FEB_OK = 0
ERRORS = {-1: "FEB_ERR_ARG", -2: "FEB_ERR_CUDA", -3: "FEB_ERR_BREAKDOWN", -4: "FEB_ERR_NAN", -5: "FEB_ERR_COARSE",
          -6: "FEB_ERR_TIMEOUT", -7: "FEB_ERR_INJECTED", -8: "FEB_ERR_NOMEM"}
MAT_ISO_SRI, MAT_ISO_FULL, MAT_ORTHO = 0, 1, 2
PREC = {"fp64": 0, "mixed": 1, "refine": 2}

EXPORTS = ["feb_default_options", "feb_create", "feb_set_rigid_groups", "feb_solve", "feb_solve_batch", "feb_apply", "feb_precondition",
           "feb_export_solution", "feb_used_nodes", "feb_destroy", "feb_accumulate_nodal", "feb_cell_stress",
           "feb_element_forces", "feb_cell_stress_noalloc", "feb_benchmark_apply", "feb_benchmark_apply_set", "feb_benchmark_smooth_set", "feb_launch_count", "feb_pool_stats", "feb_last_error",
           "feb_region_forces", "feb_rigid_fit", "feb_relative_displacement", "feb_sample_cells",
           "feb_nearest_active", "feb_sample_nodes", "feb_split_connectivity",
           "feb_mix_materials", "feb_net_conv", "feb_net_wgrad", "feb_net_colsum", "feb_net_weights", "feb_net_head",
           "feb_net_adam", "feb_net_sumsq", "feb_net_inputs", "feb_net_targets", "feb_net_to_nodes",
           "feb_net_head_grad", "feb_net_loss", "feb_net_energy_loss", "feb_label_lattice"]

GATHER_SHIFT, GATHER_DOWN, GATHER_ONE, GATHER_UP = 0, 1, 2, 3


class FebGrid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("xe", C.c_void_p), ("ye", C.c_void_p), ("ze", C.c_void_p)]


class FebOperator(C.Structure):
    _fields_ = [("mat_mode", C.c_int32), ("mat", C.c_void_p), ("active", C.c_void_p), ("cn", C.c_void_p),
                ("nnode_total", C.c_int64), ("orig", C.c_void_p), ("npen", C.c_int64), ("pen_node", C.c_void_p),
                ("pen_k", C.c_void_p), ("nextra", C.c_int64), ("extra_row", C.c_void_p), ("extra_col", C.c_void_p),
                ("extra_val", C.c_void_p), ("nmark", C.c_int64), ("mark_used", C.c_void_p)]


class FebOptions(C.Structure):
    _fields_ = [("precision", C.c_int32), ("maxiter", C.c_int32), ("tol", C.c_double), ("min_dofs", C.c_int32),
                ("max_levels", C.c_int32), ("cheb_degree", C.c_int32), ("check_every", C.c_int32),
                ("inner_tol", C.c_double), ("inner_maxiter", C.c_int32), ("use_graphs", C.c_int32),
                ("seed", C.c_uint64), ("x0_mode", C.c_int32), ("level_kernel", C.c_int32)]


class FebInfo(C.Structure):
    _fields_ = [("iters", C.c_int32), ("flag", C.c_int32), ("levels", C.c_int32), ("sweeps", C.c_int32),
                ("relres", C.c_double), ("t_setup_ms", C.c_double), ("t_solve_ms", C.c_double),
                ("ndof", C.c_int64), ("level_dofs", C.c_int64 * 8), ("lmax", C.c_double * 8),
                ("coarse_n", C.c_int32), ("kernel_launches", C.c_int32), ("ku_shape", C.c_int32 * 4),
                ("t_stage_ms", C.c_double * 8), ("x0_used", C.c_int32), ("x0_scale", C.c_float),
                ("ku_kind", C.c_int32)]


class FebNetGrid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32)]


class FebConv(C.Structure):
    _fields_ = [("gather", C.c_int32), ("scatter", C.c_int32), ("grid", FebNetGrid), ("fine", FebNetGrid),
                ("in", C.c_void_p), ("in_ld", C.c_int32), ("in_c0", C.c_int32), ("kc", C.c_int32), ("n", C.c_int32),
                ("wt", C.c_void_p), ("out", C.c_void_p), ("out_ld", C.c_int32), ("out_c0", C.c_int32),
                ("scatter_c", C.c_int32), ("relu", C.c_int32), ("bias", C.c_void_p), ("mask", C.c_void_p),
                ("mask_ld", C.c_int32), ("mask_c0", C.c_int32), ("accumulate", C.c_int32), ("pad_", C.c_int32),
                ("status", C.c_void_p)]


class FebWgrad(C.Structure):
    _fields_ = [("mode", C.c_int32), ("pad_", C.c_int32), ("grid", FebNetGrid), ("fine", FebNetGrid),
                ("p", C.c_void_p), ("p_ld", C.c_int32), ("p_c0", C.c_int32), ("na", C.c_int32),
                ("q_ld", C.c_int32), ("q_c0", C.c_int32), ("nb", C.c_int32), ("q", C.c_void_p), ("dw", C.c_void_p)]


class FebError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load():
    """Load libfeb200.so (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m comech_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    lib.feb_default_options.argtypes = [C.POINTER(FebOptions)]
    lib.feb_default_options.restype = None
    lib.feb_create.argtypes = [C.POINTER(FebGrid), C.POINTER(FebOperator), C.POINTER(FebOptions), P, C.POINTER(P)]
    lib.feb_set_rigid_groups.argtypes = [P, C.c_int32, P, P]
    lib.feb_solve.argtypes = [P, P, P, P, C.POINTER(FebInfo)]
    lib.feb_apply.argtypes = [P, C.c_int32, P, P]
    lib.feb_precondition.argtypes = [P, P, P]
    lib.feb_solve_batch.argtypes = [P, C.c_int32, P, P, P, P]
    lib.feb_label_lattice.argtypes = [P, P, C.c_int32, P, C.c_int32, P, C.c_int32, P, P]
    lib.feb_export_solution.argtypes = [P, P, P]
    lib.feb_used_nodes.argtypes = [P, C.POINTER(C.c_int64), P]
    lib.feb_destroy.argtypes = [P]
    lib.feb_accumulate_nodal.argtypes = [C.c_int64, P, P, P, P]
    lib.feb_cell_stress.argtypes = [C.POINTER(FebGrid), C.c_int32, P, P, C.c_int64, P, P, C.c_int32, P, P, P, P]
    lib.feb_cell_stress_noalloc.argtypes = lib.feb_cell_stress.argtypes
    lib.feb_element_forces.argtypes = [C.POINTER(FebGrid), P, P, C.c_int64, P, P, P, P]
    lib.feb_benchmark_apply.argtypes = [P, C.c_int32, P, P, C.c_int32, C.POINTER(C.c_float)]
    lib.feb_benchmark_apply_set.argtypes = [P, C.c_int32, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                            C.c_int32, C.POINTER(C.c_float)]
    lib.feb_benchmark_smooth_set.argtypes = [P, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                             C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32,
                                             C.POINTER(C.c_float)]
    lib.feb_region_forces.argtypes = [C.POINTER(FebGrid), P, P, P, P, P, P, C.c_int32, C.c_int32, C.c_int64, P, P, P]
    lib.feb_rigid_fit.argtypes = [P, P, C.c_int64, P, P]
    lib.feb_relative_displacement.argtypes = [C.POINTER(FebGrid), P, C.c_int64, P, P, P, P]
    lib.feb_sample_cells.argtypes = ([C.POINTER(FebGrid)] + [C.c_int32] * 4 + [P] * 9 + [P] * 5 + [P] * 4 + [P])
    lib.feb_nearest_active.argtypes = [C.POINTER(FebGrid), P, P, P]
    lib.feb_sample_nodes.argtypes = [C.POINTER(FebGrid)] + [C.c_int32] * 3 + [P] * 6 + [P] * 4 + [P]
    lib.feb_split_connectivity.argtypes = [C.POINTER(FebGrid), P, P, P, C.c_int32, P, P, C.c_int64,
                                           C.POINTER(C.c_int64), C.POINTER(C.c_int64), P]
    lib.feb_mix_materials.argtypes = [C.c_int32] * 4 + [P, C.c_int32] + [P] * 11
    lib.feb_net_conv.argtypes = [C.POINTER(FebConv), P]
    lib.feb_net_wgrad.argtypes = [C.POINTER(FebWgrad), P]
    lib.feb_net_colsum.argtypes = [P, C.c_int64, C.c_int32, C.c_int32, C.c_int32, P, P]
    lib.feb_net_weights.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int32, P]
    lib.feb_net_head.argtypes = [P, C.c_int32, C.c_int64, P, P, P, P, P, C.c_float, P, P, C.c_int32, P, P, P]
    lib.feb_net_adam.argtypes = [P, P, P, P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32,
                                 C.c_float, P]
    lib.feb_net_sumsq.argtypes = [P, C.c_int64, P, P]
    lib.feb_net_inputs.argtypes = [FebNetGrid, P, C.POINTER(FebGrid), P, P, P, C.c_int64, P, C.c_int64, P, C.c_int64,
                                   P, P, C.c_double, P, P, P]
    lib.feb_net_targets.argtypes = [FebNetGrid, P, C.c_double, P, P, P]
    lib.feb_net_to_nodes.argtypes = [FebNetGrid, P, P, C.c_double, C.POINTER(FebGrid), P, P, C.c_int64, P, P]
    lib.feb_net_head_grad.argtypes = [P, C.c_int32, C.c_int64, P, P, P, C.c_int32, P, P, P]
    lib.feb_net_loss.argtypes = [FebNetGrid, P, P, P, P, C.c_float, C.c_float, C.c_float, P, P, P]
    lib.feb_net_energy_loss.argtypes = [FebNetGrid, P, P, P, P, P, C.c_float, P, P, P]
    lib.feb_pool_stats.argtypes = [P, P, P]
    lib.feb_launch_count.argtypes = []
    lib.feb_launch_count.restype = C.c_int64
    lib.feb_last_error.argtypes = []
    lib.feb_last_error.restype = C.c_char_p
    for name in EXPORTS:
        if name not in ("feb_default_options", "feb_last_error", "feb_launch_count"):
            getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def check(code):
    if code != FEB_OK:
        raise FebError(code, load().feb_last_error().decode())


def default_options():
    o = FebOptions()
    load().feb_default_options(C.byref(o))
    return o
