"""Loader and ctypes prototypes of libpsum_b200.so (include/psum_field_solver.h,
include/psum_pic.h, include/psum_interp.h).

The library is built in-tree (``psum_b200/libpsum_b200.so``) by
``psum_b200.build.build()``.  There is no fallback: every entry point of this
package needs the CUDA library, and importing a function that needs it raises
if the library is missing.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsum_b200.so")

P = C.c_void_p
ULL = C.c_ulonglong
I = C.c_int
D = C.c_double


class FuncTable(C.Structure):
    """struct func_table (src/field_solver/register/interface.h:14-23)."""
    _fields_ = [("init", C.CFUNCTYPE(P)),
                ("set_matrix", C.CFUNCTYPE(None, P, ULL, ULL, ULL, P, P, P)),
                ("solve", C.CFUNCTYPE(None, P, P, P)),
                ("set_options", C.CFUNCTYPE(None, P, C.c_char_p)),
                ("set_source_replace", C.CFUNCTYPE(None, P, ULL, P, P)),
                ("set_source_addback", C.CFUNCTYPE(None, P, ULL, P, P)),
                ("free", C.CFUNCTYPE(None, P))]


class GridDesc(C.Structure):
    """psum_pic_grid_desc."""
    _fields_ = [("dim", I), ("cells", I * 3), ("lower", D * 3), ("upper", D * 3), ("periodic", I * 3)]


class SpeciesDesc(C.Structure):
    """psum_pic_species_desc."""
    _fields_ = [("charge", D), ("mass", D), ("weight", D)]


# Every symbol declared in include/*.h, with (restype, argtypes).
PROTOTYPES = {
    # block 1: PSuM plugin registry
    "register_solver": (None, [C.c_char_p, FuncTable]),
    "get_solver_funcs": (FuncTable, [C.c_char_p]),
    # block 2: status-returning solver API
    "psum_last_error": (C.c_char_p, []),
    "psum_kernel_launches": (C.c_ulonglong, []),
    "psum_mg_create": (I, [C.c_char_p, C.POINTER(P)]),
    "psum_mg_set_options": (I, [P, C.c_char_p]),
    "psum_mg_set_matrix": (I, [P, ULL, ULL, ULL, P, P, P]),
    "psum_mg_set_source_replace": (I, [P, ULL, P, P]),
    "psum_mg_set_source_addback": (I, [P, ULL, P, P]),
    "psum_mg_solve": (I, [P, P, P]),
    "psum_mg_solve_async": (I, [P, P, P, P]),
    "psum_mg_last_stats": (I, [P, C.POINTER(I), C.POINTER(I), C.POINTER(D), C.POINTER(D)]),
    "psum_mg_hierarchy_info": (I, [P, C.POINTER(I), C.POINTER(ULL), C.POINTER(ULL)]),
    "psum_mg_tma_sweeps": (I, [P, C.POINTER(I)]),
    "psum_mg_destroy": (I, [P]),
    # block 3: FD operator assembly
    "psum_poisson_assemble": (I, [I, P, P, P, D, ULL, P, C.POINTER(ULL), P, P, P]),
    # particle kernel set
    "psum_pic_create": (I, [C.POINTER(GridDesc), I, C.POINTER(P)]),
    "psum_pic_destroy": (I, [P]),
    "psum_pic_set_stream": (I, [P, P]),
    "psum_pic_set_options": (I, [P, C.c_char_p]),
    "psum_pic_add_species": (I, [P, C.POINTER(SpeciesDesc), ULL, C.POINTER(I)]),
    "psum_pic_load": (I, [P, I, ULL, P, P]),
    "psum_pic_load_device": (I, [P, I, ULL, P, P]),
    "psum_pic_count": (I, [P, I, C.POINTER(ULL), C.POINTER(ULL)]),
    "psum_pic_get_state": (I, [P, I, P, P]),
    "psum_pic_get_state_device": (I, [P, I, P, P]),
    "psum_pic_get_keys": (I, [P, I, P]),
    "psum_pic_sort": (I, [P]),
    "psum_pic_bin": (I, [P, I, P, P, P, P, C.POINTER(ULL)]),
    "psum_pic_deposit": (I, [P]),
    "psum_pic_rho": (I, [P, D, P]),
    "psum_pic_density": (I, [P, I, P]),
    "psum_pic_push": (I, [P, P, D, I, P]),
    "psum_pic_get_losses": (I, [P, P, I]),
    "psum_pic_join": (I, [P]),
    "psum_pic_append": (I, [P, I, ULL, P, P]),
    "psum_pic_append_device": (I, [P, I, ULL, P, P]),
    "psum_pic_step": (I, [P, P, D, P, P, D, I, P]),
    "psum_pic_set_timing": (I, [P, I]),
    "psum_pic_get_timing": (I, [P, P, P, I]),
    "psum_pic_get_phase_times": (I, [P, P, P, I, I]),
    "psum_pic_diagnostics": (I, [P, P, D, P]),
    "psum_pic_get_step_diagnostics": (I, [P, D, P]),
    "psum_pic_device_errors": (I, [P, C.POINTER(C.c_uint)]),
    "psum_pic_state_bytes": (I, [P, I, C.POINTER(ULL)]),
    "psum_pic_save_state": (I, [P, I, P]),
    "psum_pic_restore_state": (I, [P, I, P]),
    "psum_pic_adjoint_push": (I, [P, I, P, D, P, P, P]),
    "psum_pic_adjoint_deposit": (I, [P, I, P, P]),
    "psum_bin_positions_noalloc": (I, [C.POINTER(GridDesc), ULL, P, P, P, P, P, C.POINTER(ULL), P]),
    # B-spline interpolation (include/psum_interp.h)
    "psum_interp_bspline": (I, [C.POINTER(GridDesc), I, ULL, P, P, P, P, P]),
    "psum_interp_diff_bspline": (I, [C.POINTER(GridDesc), I, ULL, P, P, P, P, P]),
    "psum_add_back_bspline": (I, [C.POINTER(GridDesc), I, ULL, P, D, P, P, P, P]),
    "psum_bspline_deposit_bits": (I, [ULL, C.POINTER(I)]),
}

STATUS = {0: "PSUM_OK", 1: "PSUM_ERR_INVALID_ARGUMENT", 2: "PSUM_ERR_NOT_READY", 3: "PSUM_ERR_CUDA",
          4: "PSUM_ERR_NOT_CONVERGED", 5: "PSUM_ERR_DIVERGED", 6: "PSUM_ERR_OVERFLOW", 7: "PSUM_ERR_NONFINITE",
          8: "PSUM_ERR_INTERNAL"}


class PsumError(RuntimeError):
    """A psum_* entry point returned a non-zero psum_status."""

    def __init__(self, code, message):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


_lib = None


def lib():
    """The loaded library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libpsum_b200.so not found at {LIB_PATH}: run psum_b200.build.build() "
                              "(nvcc for sm_100a); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code):
    """Raise PsumError for a non-zero status."""
    if code != 0:
        msg = lib().psum_last_error()
        raise PsumError(code, msg.decode() if msg else "")
    return code
