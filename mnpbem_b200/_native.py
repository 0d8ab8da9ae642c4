"""ctypes binding of libbem200.so (the C ABI declared in include/bem200.h).

The library is built in-tree (``python -m mnpbem_b200.build``) and loaded from
``mnpbem_b200/lib/libbem200.so``.  There is no fallback: if the library is
missing, or a call returns a non-zero status, a RuntimeError is raised with the
library's message.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbem200.so")

C128 = 0
C64 = 1

# status codes (include/bem200.h)
ERR_SINGULAR = 3
ERR_TIMEOUT = 5
ERR_NOCONV = 6
ERR_PIVOTING = 7

_lib = None

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_dbl = ctypes.c_double
_sz = ctypes.c_size_t

# name -> (restype, argtypes)
_SIGS = {
    "bem200_version": (ctypes.c_int, []),
    "bem200_launch_count": (ctypes.c_uint64, []),
    "bem200_last_error": (ctypes.c_int, [ctypes.c_char_p, _sz]),
    "bem200_refine_count": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _dbl, _dbl, _vp, _vp]),
    "bem200_scan_i32": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp]),
    "bem200_refine_fill": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _dbl, _dbl, _vp, _vp, _vp, _vp, _vp]),
    "bem200_refine_integrals": (ctypes.c_int, [_i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                               _vp]),
    "bem200_closed_correction": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _i64, _vp,
                                                _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_refine_project": (ctypes.c_int, [_i64, _vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_green_assemble": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, _vp,
                                             _vp, _i64, _vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp,
                                             _vp, _vp, _i64, _vp]),
    "bem200_green_assemble_dk": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                                ctypes.c_int, _vp, _vp, _vp, _i64, _vp, _vp, ctypes.c_int, _vp, _vp,
                                                _vp, _vp, _vp, _vp, _i64, _vp]),
    "bem200_green_assemble_cart": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, _vp,
                                                  _vp, _i64, _vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp]),
    "bem200_green_potential": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp,
                                              _vp, _vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp,
                                              _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bem200_green_field": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                          _vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _dbl, ctypes.c_int, _vp, _vp,
                                          _vp, _vp, _vp, _vp, _vp]),
    "bem200_gemm": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                   _i64, _vp, _i64, _vp, _vp, _i64, _vp, _sz, _vp]),
    "bem200_gemm_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bem200_getrf": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _i64, _vp, _vp, _vp, _vp, _sz,
                                    _vp]),
    "bem200_getrf_ex": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _i64, _vp, _vp, _vp, _vp, _sz,
                                       ctypes.c_int, ctypes.c_int, _vp]),
    "bem200_getrf_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bem200_getrs_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bem200_getrs": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _i64, _vp, _vp,
                                    _i64, _vp, _sz, _vp, _vp, _vp]),
    "bem200_getrs_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _i64, _vp, _vp, _i64,
                                            _vp, _vp]),
    "bem200_bem_status": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_bem_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int]),
    "bem200_bem_slots": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "bem200_bem_init": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp,
                                       _dbl, _vp, _sz, _vp, _vp]),
    "bem200_bem_init_ex": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp,
                                          _dbl, _vp, _sz, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_bem_solve_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bem200_bem_solve": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp,
                                        _vp, ctypes.c_int, _vp, _vp, _vp, _dbl, _vp, _vp, _vp, _vp, _sz, _vp]),
    "bem200_bem_apply_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int]),
    "bem200_bem_apply": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp,
                                        _dbl, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bem200_bem_solve_ir": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                           ctypes.c_int, _vp, _vp, _vp, _dbl, _dbl, ctypes.c_int, _vp, _vp, _vp, _vp,
                                           _sz, _vp, _vp, _vp]),
    "bem200_inverse_nopiv_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int]),
    "bem200_inverse_nopiv": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int64, _vp, _sz,
                                            _vp, _dbl, _vp, _vp]),
    "bem200_bem_solve_ir_ex": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp,
                                              _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _dbl, _dbl, ctypes.c_int,
                                              _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp]),
    "bem200_bem_solve_T_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bem200_bem_solve_T": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                          ctypes.c_int, _vp, _vp, _vp, _dbl, _vp, _vp, _vp]),
    "bem200_bem_apply_T_workspace_size": (_sz, [ctypes.c_int, ctypes.c_int]),
    "bem200_bem_apply_T": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp,
                                          _vp, _dbl, _vp, _vp, _vp, _vp, _vp]),
    "bem200_shape_gradient_workspace_size": (_sz, [ctypes.c_int, _i64, ctypes.c_int]),
    "bem200_shape_gradient": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                             _dbl, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64, _vp, _vp, _vp, _vp, _vp,
                                             _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bem200_convert_c128_c64": (ctypes.c_int, [_i64, _vp, _vp, _vp]),
    "bem200_bem_precond": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                          ctypes.c_int, _vp, _vp, _vp, _dbl, _vp, _vp, _vp, _sz, _vp]),
    "bem200_bem_relabel": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_op_prep": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                      _vp]),
    "bem200_op_combine": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _dbl, _vp, _vp, _vp]),
    "bem200_hmat_gather_rows": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "bem200_hmat_permute": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp]),
    "bem200_hmat_pack_dense": (ctypes.c_int, [ctypes.c_int, _vp, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_hmat_aca": (ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _dbl, _vp, _vp, _vp,
                                       ctypes.c_int, ctypes.c_int, _vp]),
    "bem200_hmat_matvec": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp,
                                          _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "bem200_hmat_matvec_items": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                                _vp, _vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, _vp, _vp, _vp,
                                                ctypes.c_int, _vp, ctypes.c_int, _vp, _vp, _vp]),
    "bem200_hmat_compress_green": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int,
                                                  _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp,
                                                  ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                                  _dbl, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "bem200_planewave_rhs": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _dbl,
                                            ctypes.c_int, _vp, _vp, _vp, _vp]),
    "bem200_farfield": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _dbl, _vp,
                                       _vp, _vp, _vp, _vp]),
    "bem200_gmres_orth_workspace_size": (_sz, [ctypes.c_int]),
    "bem200_gmres_orth": (ctypes.c_int, [_i64, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "bem200_gmres_combine": (ctypes.c_int, [_i64, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    "bem200_zaxpy": (ctypes.c_int, [_i64, _vp, _vp, _vp, _vp]),
}


def lib():
    """Load libbem200.so (once).  Raises RuntimeError when it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libbem200.so not found at {} -- build it with `python -m mnpbem_b200.build`"
                               .format(LIB_PATH))
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    lib().bem200_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status, what="bem200"):
    if status != 0:
        raise RuntimeError("{} failed (status {}): {}".format(what, status, last_error()))


def call(name, *args):
    """Call ``name`` and raise RuntimeError on a non-zero status."""
    fn = getattr(lib(), name)
    check(fn(*args), name)


def ptr(t):
    """Device (or host) address of a torch tensor, or None."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
