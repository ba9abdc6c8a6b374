"""ctypes binding of libbsrgpu.so (the C ABI declared in include/bsr_b200.h).

The library is built in-tree by bsr_b200/build.py.  There is no fallback: if
the shared object is missing or fails to load, every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbsrgpu.so")

_c_long = ctypes.c_long
_c_int, _c_double, _c_char, _c_void_p, _c_size_t = (ctypes.c_int, ctypes.c_double, ctypes.c_char,
                                                     ctypes.c_void_p, ctypes.c_size_t)
_P = ctypes.c_void_p                      # device or host pointer
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)

# (name, restype, argtypes) for every symbol of include/bsr_b200.h
SIGNATURES = [
    ("bsrg_last_error", ctypes.c_char_p, []),
    ("bsrg_version", _c_int, []),
    ("bsrg_mkgrid", _c_int, [_c_int, _c_int, _c_double, _c_double, _c_double, _c_double, _DP, _c_int,
                             _IP, _IP, _IP, _DP]),
    ("bsrg_define_spline", _c_int, [_c_int, _c_int, _DP, _c_int, _c_int, _c_double, _P,
                                    ctypes.POINTER(_c_void_p)]),
    ("bsrg_basis_free", _c_int, [_P]),
    ("bsrg_basis_dims", _c_int, [_P, _IP]),
    ("bsrg_basis_get", _c_int, [_P, _c_int, _P, _P]),
    ("bsrg_mrm", _c_int, [_P, _c_int, _P, _P]),
    ("bsrg_rk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P]),
    ("bsrg_mrk_cell", _c_int, [_P, _c_int, _P, _c_int, _P]),
    ("bsrg_mrk_cell_from_moments", _c_int, [_P, _P, _P, _P, _P, _c_int, _P]),
    ("bsrg_nk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P]),
    ("bsrg_mnk_cell", _c_int, [_P, _c_int, _c_double, _P, _c_int, _P]),
    ("bsrg_mk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P]),
    ("bsrg_tk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P]),
    ("bsrg_vk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P, _P, _P]),
    ("bsrg_mvk_cell", _c_int, [_P, _c_int, _c_double, _P, _c_int, _P]),
    ("bsrg_wk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P, _P, _P]),
    ("bsrg_mwk_cell", _c_int, [_P, _c_int, _c_double, _P, _c_int, _P]),
    ("bsrg_qk_moments", _c_int, [_P, _c_int, _P, _P, _P, _P, _P, _P]),
    ("bsrg_channel_weights", _c_int, [_P, _c_int, _P, _c_int, _P, _P, _P, _P]),
    ("bsrg_mqk_cell", _c_int, [_P, _c_int, _c_double, _P, _c_int, _P]),
    ("bsrg_mtk_cell", _c_int, [_P, _c_int, _c_double, _P, _c_int, _P]),
    ("bsrg_mmk_cell", _c_int, [_P, _c_int, _c_double, _P, _c_int, _P]),
    ("bsrg_mrk_cell_noalloc", _c_int, [_P, _c_int, _P, _c_int, _P]),
    ("bsrg_density", _c_int, [_c_int, _c_int, _P, _P, _P, _c_char, _P]),
    ("bsrg_convol", _c_int, [_c_int, _c_int, _P, _P, _P, _c_int, _c_int, _c_char, _c_char, _P]),
    ("bsrg_sum_amb", _c_int, [_c_int, _c_int, _P, _P, _c_char, _P, _P]),
    ("bsrg_bav", _c_int, [_c_int, _c_int, _P, _P, _P, _c_char, _c_char, _P]),
    ("bsrg_bvmv", _c_int, [_c_int, _c_int, _P, _c_char, _P, _P, _P, _P]),
    ("bsrg_quadr", _c_int, [_P, _P, _P, _c_int, _P, _P]),
    ("bsrg_ctx_create", _c_int, [_c_int, _P, ctypes.POINTER(_c_void_p)]),
    ("bsrg_ctx_destroy", _c_int, [_P]),
    ("bsrg_ctx_workspace_bytes", _c_size_t, [_P]),
    ("bsrg_ctx_set_timing", _c_int, [_P, _c_int]),
    ("bsrg_ctx_stage_times", _c_int, [_P, _DP, _IP, _c_int]),
    ("bsrg_ctx_stage_flops", _c_int, [_P, _DP, _c_int]),
    ("bsrg_tables_create", _c_int, [_P, _P, _c_int, ctypes.POINTER(_c_void_p)]),
    ("bsrg_tables_free", _c_int, [_P]),
    ("bsrg_tables_bytes", _c_size_t, [_P]),
    ("bsrg_ctx_use_tables", _c_int, [_P, _P]),
    ("bsrg_assemble", _c_int, [_P, _P, _c_double, _c_int, _IP, _DP, _c_int, _P, _c_int, _c_int,
                               _IP, _IP, _IP, _IP, _IP, _IP, _DP, _P, _P, _P]),
    ("bsrg_add_two_electron", _c_int, [_P, _P, _c_int, _c_int, _P, _c_int, _c_int, _IP, _IP, _IP, _IP, _IP,
                                       _IP, _DP, _P, _P]),
    ("bsrg_diag_hd", _c_int, [_P, _P, _c_int, _IP, _P, _c_int, _c_int, _c_int, _c_double, _c_double,
                              _c_int, _P, _IP, _P, _P]),
    ("bsrg_diag_hd_gen", _c_int, [_P, _P, _c_int, _IP, _P, _P, _c_int, _c_int, _c_int, _c_double, _c_double,
                                  _c_int, _P, _IP, _P, _P]),
    ("bsrg_bs_orth", _c_int, [_P, _P, _c_int, _c_int, _P, _IP, _IP, _P]),
    ("bsrg_diag_hd_ipsol", _c_int, [_P, _c_int, _IP]),
    ("bsrg_ctx_set_refine", _c_int, [_P, _c_int]),
    ("bsrg_ctx_set_precision", _c_int, [_P, _c_int]),
    ("bsrg_ctx_set_eigensolver", _c_int, [_P, _c_int]),
    ("bsrg_diag_hd_refine_stats", _c_int, [_P, _c_int, _P, _P]),
    ("bsrg_ctx_channel_fallbacks", _c_int, [_P, _P]),
    ("bsrg_dgemm", _c_int, [_c_char, _c_char, _c_int, _c_int, _c_int, _c_double, _P, _c_long, _c_long, _P,
                            _c_long, _c_long, _c_double, _P, _c_long, _c_long, _c_int, _P]),
    ("bsrg_rsol_out", _c_int, [_P, _c_int, _c_int, _IP, _P, _c_int, _P, _P, _P]),
    ("bsrg_dsytrd", _c_int, [_P, _c_int, _P, _c_int, _P, _P, _P]),
    ("bsrg_dstedc", _c_int, [_P, _c_int, _P, _P, _P, _P, _c_int]),
    ("bsrg_dsyevd", _c_int, [_P, _c_int, _P, _c_int, _P, _P, _c_int]),
    ("bsrg_dsytrd_2stage", _c_int, [_P, _c_int, _P, _c_int, _P, _P]),
    ("bsrg_dgemm_tf32x3", _c_int, [_c_int, _c_int, _c_int, _c_double, _P, _c_int, _P, _c_int, _c_double, _P,
                                   _c_int, _P, _P]),
    ("bsrg_dgemm_ozaki_work_bytes", _c_size_t, [_c_int, _c_int, _c_int, _c_int]),
    ("bsrg_dgemm_ozaki", _c_int, [_c_int, _c_int, _c_int, _c_double, _P, _c_int, _P, _c_int, _c_double, _P, _c_int,
                                  _c_int, _P, _c_size_t, _P, _P]),
    ("bsrg_partial_wave_solve", _c_int, [_P, _c_int, _c_int, _DP, _c_double, _c_int, _IP, _DP, _c_int, _DP,
                                         _c_int, _c_int, _IP, _IP, _IP, _IP, _IP, _IP, _DP, _c_int, _DP, _IP]),
]

_lib = None


class BsrgError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, name, rc, msg):
        super().__init__("%s failed (status %d): %s" % (name, rc, msg))
        self.status = rc


def lib():
    """Load libbsrgpu.so once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("bsr_b200: %s is missing; run `python bsr_b200/build.py` "
                              "(or __graft_entry__.build())" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(name, rc):
    if rc != 0:
        raise BsrgError(name, rc, lib().bsrg_last_error().decode(errors="replace"))
    return rc


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))
