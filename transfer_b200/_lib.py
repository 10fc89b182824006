"""ctypes binding of libtransfer_b200.so (the C ABI in include/transfer_b200.h).

The library is built in-tree (``make -C transfer_b200/csrc``) and loaded from
this package directory.  There is no fallback: importing the package without
the built library raises ImportError.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtransfer_b200.so")

tr_idx = C.c_uint32
ABI_VERSION = 2  # TR_ABI_VERSION of the header these structures mirror

# status codes (tr_status)
TR_OK = 0
TR_ERR_INVALID_ARG = 1
TR_ERR_CUDA = 2
TR_ERR_NOT_CONVERGED = 3
TR_ERR_NAN = 4
TR_ERR_NO_DEVICE = 5
TR_ERR_MESH = 6
TR_ERR_CONFIG = 7
TR_ERR_OUT_OF_MEMORY = 8
TR_ERR_UNSUPPORTED = 9
TR_ERR_IO = 10

TR_BC_VACUUM, TR_BC_REFLECTIVE, TR_BC_INCIDENT = 0, 1, 2
TR_SURFACE_AXIS, TR_SURFACE_EXACT = 0, 1
TR_PREC_NONE, TR_PREC_REFERENCE, TR_PREC_JACOBI = 0, 1, 2
TR_MODE_FP64, TR_MODE_MIXED = 0, 1
TR_ENGINE_PERSISTENT, TR_ENGINE_GRAPH, TR_ENGINE_LAUNCH, TR_ENGINE_PERSISTENT_SR = 0, 1, 2, 3
TR_OPERATOR_SIMT, TR_OPERATOR_TENSOR = 0, 1
TR_SWEEP_GMRES, TR_SWEEP_SOURCE_ITERATION = 0, 1
TR_SWEEP_PREC_NONE, TR_SWEEP_PREC_DSA = 0, 1
TR_SWEEP_DSA_AUTO, TR_SWEEP_DSA_CLUSTER, TR_SWEEP_DSA_EVEN_PARITY = 0, 1, 2
TR_MOMENTS_TCGEN05, TR_MOMENTS_MMA_SYNC, TR_MOMENTS_TMA_FFMA2 = 0, 1, 2
TR_BATCH_RULE, TR_BATCH_STATIC_FULL, TR_BATCH_STATIC_SMALL, TR_BATCH_QUEUE_FULL, TR_BATCH_QUEUE_SMALL = -1, 0, 1, 2, 3
TR_VTK_POINT, TR_VTK_CELL = 0, 1
TR_VTK_SCALAR, TR_VTK_VECTOR, TR_VTK_TENSOR = 0, 1, 2


class tr_tetrahedron(C.Structure):
    _fields_ = [("p", tr_idx * 4), ("kappa_volume", C.c_double), ("I_p", C.c_double),
                ("s", (C.c_double * 3) * 4)]


class tr_face(C.Structure):
    _fields_ = [("p", tr_idx * 4), ("s", C.c_double * 3), ("_pad", C.c_double * 3)]


class tr_mesh_view(C.Structure):
    _fields_ = [("nP", tr_idx), ("nF", tr_idx), ("nT", tr_idx),
                ("tetstart", C.c_void_p), ("tetidx", C.c_void_p), ("tetpos", C.c_void_p),
                ("mesh", C.c_void_p),
                ("facestart", C.c_void_p), ("faceidx", C.c_void_p), ("facepos", C.c_void_p),
                ("bnd", C.c_void_p)]


class tr_angular_view(C.Structure):
    _fields_ = [("slm", tr_idx), ("omega", C.c_void_p), ("omega_pos", C.c_void_p),
                ("Ox", C.c_void_p), ("Oy", C.c_void_p), ("Oz", C.c_void_p)]


class tr_physics_view(C.Structure):
    _fields_ = [("kappa_abs_volume", C.c_void_p), ("face_bc", C.c_void_p),
                ("face_incident", C.c_void_p), ("surface_mode", C.c_int32)]


class tr_ctx_info(C.Structure):
    _fields_ = [("nP", tr_idx), ("nT", tr_idx), ("nF", tr_idx), ("slm", tr_idx), ("aslm", tr_idx),
                ("aslm_f32", tr_idx), ("n_edges", C.c_uint64), ("n_bnd_edges", C.c_uint64),
                ("device_bytes", C.c_uint64), ("device", C.c_int)]


class tr_solve_opts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("precondition", C.c_int32), ("max_iter", C.c_int32),
                ("relative", C.c_int32), ("tol", C.c_double), ("inner_tol", C.c_double),
                ("inner_max_iter", C.c_int32), ("max_outer", C.c_int32), ("engine", C.c_int32),
                ("history_len", C.c_int32), ("history", C.POINTER(C.c_double))]


class tr_solve_report(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("inner_iterations", C.c_int32),
                ("outer_steps", C.c_int32), ("lhs_applications_f64", C.c_int64),
                ("lhs_applications_f32", C.c_int64), ("diag_applications", C.c_int64),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("rhs_norm", C.c_double), ("device_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("cg_kernel_ms", C.c_double), ("cg_kernel_launches", C.c_int64)]


class tr_region_params(C.Structure):
    _fields_ = [("nreg", C.c_int32), ("kappa", C.c_void_p), ("Ip", C.c_void_p), ("albedo", C.c_void_p)]


class tr_kuhn_params(C.Structure):
    _fields_ = [("n", C.c_int32 * 3), ("box", C.c_double * 6), ("jitter", C.c_double),
                ("seed", C.c_uint64), ("region_kind", C.c_int32), ("region_arg", C.c_double * 4),
                ("ball", C.c_int32), ("ball_center", C.c_double * 3), ("ball_radius", C.c_double)]


class tr_ordinates_view(C.Structure):
    _fields_ = [("nq", C.c_uint32), ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p), ("w", C.c_void_p)]


class tr_sweep_info(C.Structure):
    _fields_ = [("nT", C.c_uint32), ("nF", C.c_uint32), ("nq", C.c_uint32), ("n_extra", C.c_uint64),
                ("n_reflective", C.c_uint32), ("n_lag", C.c_uint32), ("max_levels", C.c_uint32),
                ("forced_levels", C.c_uint32), ("device_bytes", C.c_uint64), ("device", C.c_int)]


class tr_sweep_opts(C.Structure):
    _fields_ = [("method", C.c_int32), ("mode", C.c_int32), ("tol", C.c_double), ("max_iter", C.c_int32),
                ("restart", C.c_int32), ("inner_tol", C.c_double), ("max_outer", C.c_int32),
                ("precondition", C.c_int32), ("precond_tol", C.c_double), ("precond_engine", C.c_int32)]


class tr_vtk_field(C.Structure):
    _fields_ = [("name", C.c_char_p), ("location", C.c_int32), ("kind", C.c_int32), ("data", C.c_void_p)]


class tr_sweep_report(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("outer_steps", C.c_int32),
                ("sweeps_f32", C.c_int64), ("sweeps_f64", C.c_int64), ("residual", C.c_double),
                ("rhs_norm", C.c_double), ("device_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("precond_solves", C.c_int32), ("precond_iterations", C.c_int32)]


P = C.c_void_p
D = C.c_double
I = C.c_int
S = C.c_int  # tr_status

# (name, restype, argtypes) of every exported entry point
PROTOTYPES = [
    ("tr_abi_version", I, []),
    ("tr_status_string", C.c_char_p, [S]),
    ("tr_last_error", C.c_char_p, [P]),
    ("tr_ctx_create", S, [I, C.POINTER(tr_mesh_view), C.POINTER(tr_angular_view), C.POINTER(P)]),
    ("tr_ctx_create_ex", S, [I, C.POINTER(tr_mesh_view), C.POINTER(tr_angular_view),
                             C.POINTER(tr_physics_view), C.POINTER(P)]),
    ("tr_ctx_destroy", S, [P]),
    ("tr_ctx_info_get", S, [P, C.POINTER(tr_ctx_info)]),
    ("tr_ctx_set_operator", S, [P, I]),
    ("tr_ctx_autotune_operator", S, [P, I, P]),
    ("tr_ctx_get_operator", S, [P, P]),
    ("tr_ctx_set_stream", S, [P, P]),
    ("tr_compute_lhs", S, [P, P, P]),
    ("tr_compute_lhs_diag", S, [P, P, P]),
    ("tr_compute_rhs", S, [P, P]),
    ("tr_scale", S, [P, P, D]),
    ("tr_add_prod", S, [P, P, P, D]),
    ("tr_mul_add", S, [P, P, D, P]),
    ("tr_mul_add_prod", S, [P, P, D, P, D]),
    ("tr_norm", S, [P, P, C.POINTER(D)]),
    ("tr_dot", S, [P, P, P, C.POINTER(D)]),
    ("tr_dot_noalloc", S, [P, P, C.c_uint32, C.c_uint32, C.c_uint32, P, P]),
    ("tr_compute_lhs_f32", S, [P, P, P]),
    ("tr_compute_lhs_diag_f32", S, [P, P, P]),
    ("tr_compute_rhs_f32", S, [P, P]),
    ("tr_dot_f32", S, [P, P, P, C.POINTER(D)]),
    ("tr_solve_opts_default", None, [C.POINTER(tr_solve_opts)]),
    ("tr_solve", S, [P, C.POINTER(tr_solve_opts), P, P, C.POINTER(tr_solve_report)]),
    ("tr_solve_host", S, [P, C.POINTER(tr_solve_opts), P, P, C.POINTER(tr_solve_report)]),
    ("tr_bench_lhs", S, [P, I, P, P, I, C.POINTER(D)]),
    ("tr_selftest_grid_barrier", S, [I, I, I, C.c_uint, C.POINTER(I)]),
    ("tr_compute_moments", S, [P, P, P, P]),
    ("tr_compute_flux", S, [P, P, P]),
    ("tr_eig_lanczos", S, [P, P, P, P, I, C.POINTER(D), C.POINTER(D), C.POINTER(I)]),
    ("tr_trieig", D, [P, P, I]),
    ("tr_angular_create", S, [I, C.POINTER(P)]),
    ("tr_angular_view_get", S, [P, C.POINTER(tr_angular_view)]),
    ("tr_angular_destroy", None, [P]),
    ("tr_spherical_value", D, [I, I, D, D, D]),
    ("tr_hemiquad", I, [I, P, P, P, P, I]),
    ("tr_lebedev", I, [I, P, P, P, P, I]),
    ("tr_config_load", S, [C.c_char_p, C.POINTER(P)]),
    ("tr_config_destroy", None, [P]),
    ("tr_config_get_int", I, [P, C.c_char_p, C.POINTER(I)]),
    ("tr_config_get_double", D, [P, C.c_char_p, C.POINTER(I)]),
    ("tr_config_get_string", C.c_char_p, [P, C.c_char_p]),
    ("tr_config_num_regions", I, [P]),
    ("tr_config_region_double", D, [P, I, C.c_char_p, C.POINTER(I)]),
    ("tr_meshdata_from_tets", S, [tr_idx, P, tr_idx, P, P, C.POINTER(tr_region_params), C.POINTER(P)]),
    ("tr_meshdata_kuhn", S, [C.POINTER(tr_kuhn_params), C.POINTER(tr_region_params), C.POINTER(P)]),
    ("tr_meshdata_view_get", S, [P, C.POINTER(tr_mesh_view)]),
    ("tr_meshdata_coords", P, [P]),
    ("tr_meshdata_regions", P, [P]),
    ("tr_meshdata_kappa_abs_volume", P, [P]),
    ("tr_meshdata_face_side", P, [P]),
    ("tr_meshdata_destroy", None, [P]),
    ("tr_meshdata_read_vol", S, [C.c_char_p, C.POINTER(tr_region_params), C.POINTER(P)]),
    ("tr_meshdata_face_bcnr", P, [P]),
    ("tr_vtk_write", S, [C.c_char_p, P, I, I, P]),
    ("tr_ordinates_product", S, [I, I, P, P, P, P]),
    ("tr_sweep_create", S, [I, C.POINTER(tr_mesh_view), C.POINTER(tr_physics_view), C.POINTER(tr_ordinates_view),
                            C.POINTER(P)]),
    ("tr_sweep_destroy", S, [P]),
    ("tr_sweep_last_error", C.c_char_p, [P]),
    ("tr_sweep_info_get", S, [P, C.POINTER(tr_sweep_info)]),
    ("tr_sweep_levels", S, [P, P]),
    ("tr_sweep_apply", S, [P, I, P, P, I, P, P]),
    ("tr_sweep_psi", S, [P, P]),
    ("tr_sweep_moments", S, [P, I, P]),
    ("tr_sweep_set_moments_kernel", S, [P, I]),
    ("tr_sweep_create_group", S, [P, P, P, P, P]),
    ("tr_sweep_release_work", S, [P]),
    ("tr_sweep_set_batch_form", S, [P, I]),
    ("tr_sweep_autotune_batch", S, [I, P, I, P, P]),
    ("tr_sweep_balance", S, [P, P, P, P, P]),
    ("tr_sweep_opts_default", None, [C.POINTER(tr_sweep_opts)]),
    ("tr_sweep_solve", S, [P, C.POINTER(tr_sweep_opts), P, P, C.POINTER(tr_sweep_report)]),
    ("tr_sweep_enable_dsa", S, [P, C.POINTER(tr_mesh_view), C.POINTER(tr_physics_view)]),
    ("tr_sweep_set_coefficients", S, [P, P, P, P]),
    ("tr_sweep_apply_batch", S, [I, P, I, P, P, I, P, P]),
    ("tr_sweep_solve_batch", S, [I, P, I, D, I, P, P, P, P]),
    ("tr_sweep_autotune", S, [P, P, P]),
    ("tr_sweep_outflow", S, [P, P, C.POINTER(D)]),
    ("tr_sweep_gradient", S, [P, P, I, P, P, P, P, P]),
    ("tr_sweep_bench", S, [P, I, I, C.POINTER(D)]),
]


class TransferError(RuntimeError):
    """A tr_* call returned a non-zero tr_status."""

    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `make -C transfer_b200/csrc` "
            "(this package has no CPU fallback)")
    lib = C.CDLL(path)
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.tr_abi_version() != ABI_VERSION:
        raise ImportError(f"{path} has ABI version {lib.tr_abi_version()}, this binding expects {ABI_VERSION}: "
                          "rebuild it with `make -C transfer_b200/csrc`")
    return lib


lib = load()


def check(status, ctx=None):
    if status != TR_OK:
        msg = lib.tr_last_error(ctx)
        msg = msg.decode() if msg else lib.tr_status_string(status).decode()
        raise TransferError(status, msg)
    return status
