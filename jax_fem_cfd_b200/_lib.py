"""ctypes binding of libfemb200.so (the C ABI declared in include/fem_b200.h).

The library is the only compute path: importing works anywhere, but every
compute call requires the built library and a CUDA device and raises otherwise
(there is no CPU fallback)."""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfemb200.so")

c_int, c_double, c_void_p, c_longlong = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong
P = c_void_p  # device pointer / stream / handle

FEM_KIND_Q1_2D, FEM_KIND_Q2_2D, FEM_KIND_HEX8 = 0, 1, 2
SHAPE_QUAD4, SHAPE_QUAD9, SHAPE_HEX8, SHAPE_LIN2, SHAPE_LIN3 = 0, 1, 2, 3, 4
PREC = {None: 0, "none": 0, "jacobi": 1, "approx_inv": 2, "approx_inv_pt": 3, "multigrid": 4}
STATUS_BARRIER_TIMEOUT, STATUS_NONFINITE, STATUS_MAXITER, STATUS_BREAKDOWN = 1, 2, 4, 8
PRECISION = {"fp64": 0, "mixed": 1}


class MeshDesc(ctypes.Structure):
    _fields_ = [("kind", c_int), ("periodic", c_int), ("nex", c_int), ("ney", c_int), ("nez", c_int),
                ("lx", c_double), ("ly", c_double), ("lz", c_double)]


# name -> (restype, argtypes); mirrors include/fem_b200.h
SIGNATURES = {
    "fem_mesh_counts": (c_int, [P, P, P, P]),
    "fem_mesh_generate": (c_int, [P, P, P, P]),
    "fem_shape_functions": (c_int, [c_int, P, P, P, P, P]),
    "fem_ctx_create": (c_int, [P, c_int, P]),
    "fem_ctx_destroy": (None, [P]),
    "fem_ctx_dims": (c_int, [P, P, P, P, P, P]),
    "fem_ctx_element_data": (c_int, [P, P, P, P, P, P, P, P, P, P]),
    "fem_ctx_set_bc": (c_int, [P, P, P, c_int, P]),
    "fem_ctx_setup_multigrid": (c_int, [P, c_int, P, c_double, P]),
    "fem_ctx_level_info": (c_int, [P, c_int, P, P, P, P, P]),
    "fem_ebe_apply": (c_int, [P, c_int, P, P, c_double, P, c_double, P, c_int, c_double, P, P]),
    "fem_grad_apply": (c_int, [P, P, P, P, P]),
    "fem_div_apply": (c_int, [P, P, P, P, P]),
    "fem_convection_build": (c_int, [P, P, c_double, P, P, P, P, P]),
    "fem_ctau_tilde_build": (c_int, [P, P, P, P, P, P, P]),
    "fem_supg_tau": (c_int, [P, P, P, P, c_double, c_double, c_double, P, P, P]),
    "fem_conv_vjp": (c_int, [P, c_int, P, P, c_double, P, P]),
    "fem_transport_vjp": (c_int, [P, P, P, P, P, P, c_double, c_double, c_int, P, P, P]),
    "fem_transport_elements": (c_int, [P, P, P, c_double, c_double, c_int, c_int, P, P, P]),
    "fem_pack_create": (c_int, [P, c_int, P, P, P, P, P, P, c_double, c_int, P]),
    "fem_pack_step": (c_int, [P, P, P, P, P, P]),
    "fem_pack_info": (c_int, [P, P, P, P]),
    "fem_pack_destroy": (c_int, [P]),
    "fem_element_matrices": (c_int, [c_int, c_int, c_int, P, P, P, P, P, P, P, P]),
    "fem_assemble_diag": (c_int, [P, P, P, c_int, P, P, P]),
    "fem_lattice_interpolate": (c_int, [c_int, c_int, c_int, c_int, c_int, P, P, P]),
    "fem_lattice_restrict": (c_int, [c_int, c_int, c_int, c_int, c_int, P, P, P]),
    "fem_mg_vcycle": (c_int, [P, P, P, P]),
    "fem_pressure_solve": (c_int, [P, P, P, c_double, c_double, c_int, c_int, c_int, c_int, P, P, P]),
    "fem_bicgstab_solve": (c_int, [P, c_int, c_double, P, c_double, P, c_double, P, P, P, P, c_double, c_double,
                                   c_int, P, P, P]),
    "fem_step4": (c_int, [P, P, P, c_double, c_double, c_double, P, P, P, c_double, c_int, P, P, P, P, P]),
    "fem_transport_phi": (c_int, [P, P, P, P, c_double, c_double, c_int, P, P, c_double, P, P, P, P]),
    "fem_boundary_flux": (c_int, [P, P, P, c_int, c_int, P, P, P]),
    "fem_boundary_flux_noalloc": (c_int, [P, P, P, c_int, c_int, P, P, P]),
    "fem_boundary_flux_skipped": (c_int, [P, P, P]),
    "fem_scatter": (c_int, [P, P, c_double, c_int, P, P]),
    "fem_make_mask": (c_int, [P, c_int, c_int, P, P]),
    "fem_dot": (c_int, [P, P, P, c_int, P, P]),
    "fem_axpby": (c_int, [P, c_double, P, c_double, P, c_int, P]),
    "fem_ctx_enable_timing": (c_int, [P, c_int]),
    "fem_ctx_stage_times": (c_int, [P, P, c_int]),
    "fem_ctx_set_trace": (c_int, [P, P, c_int]),
    "fem_ctx_set_max_ctas": (c_int, [P, c_int, P]),
    "fem_ctx_set_precision": (c_int, [P, c_int, c_int, c_int]),
    "fem_selftest_barrier_timeout": (c_int, [P, P, P]),
    "fem_pressure_solve_mixed": (c_int, [P, P, P, c_double, c_int, c_int, P, P, P]),
    "fem_step4_graph": (c_int, [P, P, P, P, P, c_double, c_double, c_double, P, P, P, c_double, c_int, c_int, P, P,
                                P]),
    "fem_graph_launch": (c_int, [P, P]),
    "fem_graph_destroy": (c_int, [P]),
    "fem_launch_count": (c_longlong, []),
    "fem_last_error": (ctypes.c_char_p, []),
}

_LIB = None


class FemError(RuntimeError):
    pass


def load():
    """Load libfemb200.so and declare its signatures (no CUDA call)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FemError(f"{LIB_PATH} is not built; run `python -m jax_fem_cfd_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def check(rc, what=""):
    if rc != 0:
        msg = load().fem_last_error()
        raise FemError(f"{what} failed with status {rc}: {msg.decode() if msg else ''}")


def call(name, *args):
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc


def launch_count():
    return int(load().fem_launch_count())
