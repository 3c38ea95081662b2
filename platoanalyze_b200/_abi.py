"""ctypes binding of libpa_b200.so (the C ABI declared in include/pa_b200.h).

There is no fallback: if the shared library is missing or cannot be loaded,
load() raises, and every call into the package fails loudly.
"""
import ctypes as ct
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpa_b200.so")

P = ct.c_void_p
I32, I64, F64 = ct.c_int32, ct.c_int64, ct.c_double

PA_OK = 0
PA_ERR_INVALID_ARG = 1
STATUS_NAMES = {0: "PA_OK", 1: "PA_ERR_INVALID_ARG", 2: "PA_ERR_CUDA", 3: "PA_ERR_NOT_CONVERGED",
                4: "PA_ERR_BREAKDOWN", 5: "PA_ERR_NONFINITE", 6: "PA_ERR_NO_DEVICE", 7: "PA_ERR_UNSUPPORTED"}
PA_CONTROL_NODAL, PA_CONTROL_CELL = 0, 1
PA_FP64, PA_FP32 = 0, 1
PA_SOLVER_PCG_FP64, PA_SOLVER_PCG_MIXED, PA_SOLVER_FCG_LEARNED, PA_SOLVER_PCG_MG = 0, 1, 2, 3
PA_MG_COARSE_AUTO, PA_MG_COARSE_CHEBYSHEV = 0, 1


class ElasticParams(ct.Structure):
    _fields_ = [("youngs_modulus", F64), ("poissons_ratio", F64), ("simp_exponent", F64), ("simp_min", F64),
                ("control_layout", I32)]


class SolveOptions(ct.Structure):
    _fields_ = [("method", I32), ("rel_tol", F64), ("max_iters", I32), ("check_every", I32),
                ("use_initial_guess", I32), ("mg_coarse_solver", I32)]


class SolveStats(ct.Structure):
    _fields_ = [("iterations", I32), ("replacements", I32), ("rel_residual", F64), ("seconds", F64),
                ("converged", I32), ("kernel_launches", I64), ("fallback_iterations", I32)]


class J2Params(ct.Structure):
    _fields_ = [("youngs_modulus", F64), ("poissons_ratio", F64), ("initial_yield_stress", F64),
                ("hardening_modulus_isotropic", F64), ("hardening_modulus_kinematic", F64),
                ("elastic_penalty_exponent", F64), ("elastic_min_ersatz", F64),
                ("plastic_penalty_exponent", F64), ("plastic_min_ersatz", F64)]


class J2SolveOptions(ct.Structure):
    _fields_ = [("steps", I32), ("max_newton", I32), ("newton_tol", F64), ("adaptive_forcing", I32)]


class J2Stats(ct.Structure):
    _fields_ = [("steps", I32), ("newton_iterations", I32), ("cg_iterations", I64), ("seconds", F64),
                ("final_rel_residual", F64), ("converged", I32), ("linear_unconverged", I32),
                ("line_search_halvings", I32)]


class UpParams(ct.Structure):
    _fields_ = [("youngs_modulus", F64), ("poissons_ratio", F64), ("penalty_exponent", F64), ("penalty_min", F64),
                ("pressure_scaling", F64)]


class PcTrainOptions(ct.Structure):
    _fields_ = [("steps", I32), ("batch", I32), ("learning_rate", F64), ("seed", ct.c_uint64)]


class PcTrainStats(ct.Structure):
    _fields_ = [("initial_loss", F64), ("final_loss", F64), ("seconds", F64), ("steps", I32),
                ("kernel_launches", I64)]


# (name, restype, argtypes) for every symbol of include/pa_b200.h
SIGNATURES = [
    ("pa_version", ct.c_char_p, []),
    ("pa_last_error", ct.c_char_p, []),
    ("pa_mesh_create", I32, [P, I64, P, I64, P]),
    ("pa_mesh_create_box", I32, [I32, I32, I32, F64, F64, F64, P]),
    ("pa_mesh_destroy", I32, [P]),
    ("pa_mesh_sizes", I32, [P, P, P, P, P]),
    ("pa_mesh_get", I32, [P, P, P]),
    ("pa_mesh_graph", I32, [P, P, P]),
    ("pa_mesh_set_graph", I32, [P, P, P, I64]),
    ("pa_mesh_boundary_faces", I32, [P, I32, F64, P, P]),
    ("pa_problem_create", I32, [P, ct.POINTER(ElasticParams), P, P]),
    ("pa_problem_destroy", I32, [P]),
    ("pa_problem_add_traction", I32, [P, P, I64, P]),
    ("pa_problem_clear_tractions", I32, [P]),
    ("pa_problem_set_dirichlet", I32, [P, P, P, I64]),
    ("pa_vf_value", I32, [P, P, P, P]),
    ("pa_vf_gradient_u", I32, [P, P, P, P]),
    ("pa_vf_gradient_z", I32, [P, P, P, P]),
    ("pa_vf_gradient_x", I32, [P, P, P, P]),
    ("pa_sf_value", I32, [P, P, P, P]),
    ("pa_sf_gradient_u", I32, [P, P, P, P]),
    ("pa_sf_gradient_z", I32, [P, P, P, P]),
    ("pa_sf_gradient_x", I32, [P, P, P, P]),
    ("pa_sf_value_noalloc", I32, [P, I64, P, I64, P, P, ct.POINTER(ElasticParams), P, P]),
    ("pa_apply", I32, [P, P, P, P, I32, I32]),
    ("pa_apply_block_constraints", I32, [P, P, P, F64]),
    ("pa_solve_options_default", I32, [ct.POINTER(SolveOptions)]),
    ("pa_solve", I32, [P, P, P, P, ct.POINTER(SolveOptions), ct.POINTER(SolveStats)]),
    ("pa_problem_solution", I32, [P, P, P, ct.POINTER(SolveOptions), ct.POINTER(SolveStats)]),
    ("pa_problem_criterion_gradient", I32, [P, P, P, P, I32, ct.POINTER(SolveOptions)]),
    ("pa_time_cg_apply", I32, [P, P, I32, I32, P, P]),
    ("pa_time_apply", I32, [P, P, I32, I32, P, P]),
    ("pa_j2_radial_return", I32, [P, ct.POINTER(J2Params), P, P, P, P]),
    ("pa_j2_local_residual", I32, [P, ct.POINTER(J2Params), P, P, P, P, P]),
    ("pa_j2_solve", I32, [P, ct.POINTER(J2Params), P, ct.POINTER(J2SolveOptions), ct.POINTER(SolveOptions), P, P,
                          ct.POINTER(J2Stats)]),
    ("pa_pc_create", I32, [I32, I32, I32, ct.c_uint64, P]),
    ("pa_pc_destroy", I32, [P]),
    ("pa_pc_num_params", I32, [P, P]),
    ("pa_pc_get_params", I32, [P, P]),
    ("pa_pc_set_params", I32, [P, P]),
    ("pa_pc_forward", I32, [P, P, P]),
    ("pa_pc_backward", I32, [P, P, P, P]),
    ("pa_pc_time_forward", I32, [P, I32, P, P]),
    ("pa_pc_apply", I32, [P, P, P, P, P]),
    ("pa_pc_train", I32, [P, P, I32, P, I32, P, P, P, ct.POINTER(PcTrainOptions), ct.POINTER(PcTrainStats)]),
    ("pa_problem_set_preconditioner", I32, [P, P]),
    ("pa_boxmg_coarse_grid", I32, [P, P]),
    ("pa_boxmg_coarse_features", I32, [P, P, P]),
    ("pa_boxmg_coarse_sensitivity", I32, [P, P, P, I32, P, P, ct.POINTER(F64), P]),
    ("pa_problem_set_coarse_network", I32, [P, P]),
    ("pa_exodus_open", I32, [ct.c_char_p, ct.POINTER(P)]),
    ("pa_exodus_sizes", I32, [P, ct.POINTER(I64), ct.POINTER(I64), ct.POINTER(I32)]),
    ("pa_exodus_mesh", I32, [P, P, P]),
    ("pa_exodus_node_set", I32, [P, I32, ct.c_char_p, I32, ct.POINTER(I64), P]),
    ("pa_exodus_close", None, [P]),
    ("pa_up_residual", I32, [P, ct.POINTER(UpParams), P, P, P, I32, P, P, I32]),
    ("pa_up_solve", I32, [P, ct.POINTER(UpParams), ct.POINTER(J2Params), P, ct.POINTER(J2SolveOptions),
                          ct.POINTER(SolveOptions), P, P, P, ct.POINTER(J2Stats)]),
    ("pa_up_elastic_work", I32, [P, ct.POINTER(UpParams), ct.POINTER(J2Params), F64, F64, P, ct.POINTER(J2SolveOptions),
                                 ct.POINTER(SolveOptions), ct.POINTER(F64), P, P, P, ct.POINTER(J2Stats)]),
    ("pa_mesh_set_parts", I32, [P, I32, P]),
    ("pa_mesh_uniform_geometry", I32, [P, I32, P]),
    ("pa_mesh_box_kernels", I32, [P, I32, P]),
    ("pa_write_vtu", I32, [P, ct.c_char_p, P, P, I32]),
    ("pa_problem_part_stats", I32, [P, P, P]),
    ("pa_problem_autotune_tiles", I32, [P, P, P, P]),
]

_lib = None


class PaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load():
    """Load libpa_b200.so and bind every entry point (raises if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libpa_b200.so not built at {LIB_PATH}; run python -m platoanalyze_b200.build")
        lib = ct.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status, allow=()):
    if status != PA_OK and status not in allow:
        raise PaError(status, load().pa_last_error().decode())
    return status
