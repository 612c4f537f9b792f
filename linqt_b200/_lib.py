"""ctypes binding of liblinqt_gpu.so (the C ABI declared in include/linqt_gpu.h).

Loading fails loudly when the library has not been built: there is no CPU
fallback anywhere in this package.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblinqt_gpu.so")

c_int, c_long, c_double, c_void_p = ctypes.c_int, ctypes.c_long, ctypes.c_double, ctypes.c_void_p
P_int = ctypes.POINTER(ctypes.c_int)
P_long = ctypes.POINTER(ctypes.c_long)
P_double = ctypes.POINTER(ctypes.c_double)

ERRORS = {
    -1: "LINQT_ERR_INVALID",
    -2: "LINQT_ERR_CUDA",
    -3: "LINQT_ERR_NOMEM",
    -4: "LINQT_ERR_UNSUPPORTED",
    -5: "LINQT_ERR_INTERNAL",
    -6: "LINQT_ERR_TIMEOUT",
    -7: "LINQT_ERR_CANCELLED",
}


class LinqtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("precision", c_int), ("format", c_int), ("block_width", c_int), ("doubling", c_int),
                ("use_graphs", c_int), ("step_launches", c_int), ("realisations", c_int), ("operator_precision", c_int),
                ("thread_shape", c_int), ("reserved", c_int * 7)]


class Request(ctypes.Structure):
    _fields_ = [("kind", c_int), ("H", c_void_p), ("op", c_void_p), ("states", P_double), ("R", c_int),
                ("M", c_int), ("precision", c_int), ("mu_out", P_double), ("seed", ctypes.c_ulonglong),
                ("sigma_out", P_double), ("nump", c_int), ("band_width", ctypes.c_double),
                ("band_center", ctypes.c_double)]


# name -> (restype, argtypes)
SIGNATURES = {
    "linqt_abi_version": (c_int, []),
    "linqt_random_phase_states_dev": (c_int, [c_void_p, c_int, c_int, ctypes.c_ulonglong, c_void_p]),
    "linqt_last_error": (ctypes.c_char_p, []),
    "linqt_session_create": (c_int, [c_int, ctypes.POINTER(c_void_p)]),
    "linqt_session_destroy": (c_int, [c_void_p]),
    "linqt_session_set_stream": (c_int, [c_void_p, c_void_p]),
    "linqt_session_get_stream": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
    "linqt_session_synchronize": (c_int, [c_void_p]),
    "linqt_session_trim": (c_int, [c_void_p]),
    "linqt_session_phase_times": (c_int, [c_void_p, P_double, P_long, c_int]),
    "linqt_session_enable_timing": (c_int, [c_void_p, c_int]),
    "linqt_session_graph_stats": (c_int, [c_void_p, P_int, P_long]),
    "linqt_csr_create": (c_int, [c_void_p, c_int, P_int, P_int, P_double, c_int, ctypes.POINTER(c_void_p)]),
    "linqt_op_destroy": (c_int, [c_void_p]),
    "linqt_op_info": (c_int, [c_void_p, P_int, P_long]),
    "linqt_op_tuned": (c_int, [c_void_p, ctypes.c_char_p, c_long, P_long]),
    "linqt_op_rescale": (c_int, [c_void_p, P_double, P_double]),
    "linqt_op_multiply": (c_int, [c_void_p, c_void_p, P_double, P_double, P_double, P_double, c_int]),
    "linqt_spectral_bounds": (c_int, [c_void_p, c_void_p, P_double, P_double]),
    "linqt_moments1d": (c_int, [c_void_p, c_void_p, c_void_p, P_double, c_int, c_int, ctypes.POINTER(Opts),
                                P_double]),
    "linqt_moments1d_realisations": (c_int, [c_void_p, ctypes.POINTER(c_void_p), c_int, P_double, c_int, c_int,
                                             ctypes.POINTER(Opts), P_double]),
    "linqt_moments1d_realisations_dev": (c_int, [c_void_p, ctypes.POINTER(c_void_p), c_int, c_void_p, c_int, c_int,
                                                 ctypes.POINTER(Opts), c_void_p]),
    "linqt_moments1d_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, ctypes.POINTER(Opts),
                                    c_void_p]),
    "linqt_moments2d": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, P_double, c_int, c_int,
                                ctypes.POINTER(Opts), P_double]),
    "linqt_time_correlation_from_moments": (c_int, [c_void_p, P_double, c_int, c_int, c_int, c_double, c_double,
                                                    c_double, c_double, c_double, P_double, P_double, P_int]),
    "linqt_moments_td": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, P_double, c_int, c_int, c_int, c_double,
                                 c_double, c_double, ctypes.POINTER(Opts), P_double]),
    "linqt_moments_td_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                     c_double, c_double, c_double, ctypes.POINTER(Opts), c_void_p]),
    "linqt_moments2d_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                    ctypes.POINTER(Opts), c_void_p]),
    "linqt_kubo_fft": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, P_double, c_int, c_int, c_int, c_int,
                               c_double, c_double, ctypes.POINTER(Opts), P_double, P_double, P_double]),
    "linqt_kubo_fft_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_int,
                                   c_double, c_double, ctypes.POINTER(Opts), c_void_p]),
    "linqt_kubo_bastin": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, P_double, c_int, c_int, c_int, c_double,
                                  c_double, ctypes.POINTER(Opts), P_double, P_double, P_double, P_double]),
    "linqt_kubo_bastin_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                      c_double, c_double, ctypes.POINTER(Opts), c_void_p, c_void_p]),
    "linqt_session_set_sm_share": (c_int, [c_void_p, ctypes.c_double]),
    "linqt_session_inject_barrier_timeout": (c_int, [c_void_p, c_int, ctypes.c_longlong]),
    "linqt_moments1d_nonorth": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, P_double, c_int, c_int, c_double,
                                        c_int, ctypes.POINTER(Opts), P_double, P_long]),
    "linqt_moments1d_nonorth_dev": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                            c_double, c_int, ctypes.POINTER(Opts), c_void_p, P_long]),
    "linqt_moments1d_noalloc": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "linqt_dos_from_moments": (c_int, [c_void_p, P_double, c_int, c_int, c_double, c_double, c_double, P_double,
                                       P_double, P_int]),
    "linqt_spectral_function_from_moments": (c_int, [c_void_p, P_double, c_int, c_int, c_double, c_double, c_double,
                                                     c_int, c_int, P_double, P_double, P_int]),
    "linqt_bastin_from_moments": (c_int, [c_void_p, P_double, c_int, c_int, c_int, c_double, c_double, c_double,
                                          c_double, c_int, P_double, P_double, P_int]),
    "linqt_kubo_from_moments": (c_int, [c_void_p, P_double, c_int, c_int, c_int, c_double, c_double, c_double, c_int,
                                        c_int, c_double, c_int, P_double, P_double, P_int]),
    "linqt_jackson1d": (c_int, [P_double, c_int, c_double, c_double, P_int]),
    "linqt_jackson2d": (c_int, [P_double, c_int, c_int, c_double, c_double, c_double, P_int, P_int]),
    "linqt_locality_order": (c_int, [c_int, P_int, P_int, c_int, P_int]),
    "linqt_server_create": (c_int, [c_int, ctypes.c_size_t, c_int, ctypes.POINTER(c_void_p)]),
    "linqt_server_submit": (c_int, [c_void_p, ctypes.POINTER(Request), P_long]),
    "linqt_server_poll": (c_int, [c_void_p, c_long, P_int, P_double]),
    "linqt_server_wait_all": (c_int, [c_void_p]),
    "linqt_server_release": (c_int, [c_void_p, c_long]),
    "linqt_server_cancel": (c_int, [c_void_p, c_long]),
    "linqt_server_stats": (c_int, [c_void_p, P_long, P_long]),
    "linqt_server_destroy": (c_int, [c_void_p]),
    "linqt_tbmodel_load": (c_int, [ctypes.c_char_p, ctypes.POINTER(c_void_p)]),
    "linqt_tbmodel_destroy": (c_int, [c_void_p]),
    "linqt_tbmodel_info": (c_int, [c_void_p, P_int, P_long]),
    "linqt_supercell_csr": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, P_int, P_int, P_long, P_int, P_int, P_double,
                                    c_long]),
    "linqt_supercell_csr_dev": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, P_int, P_int, P_long, c_void_p, c_void_p,
                                        c_void_p, c_long]),
    "linqt_supercell_write_csr": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, P_int, ctypes.c_char_p]),
    "linqt_supercell_operator": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, P_int, ctypes.POINTER(c_void_p)]),
}

_lib = None


ABI_VERSION = 3  # LINQT_ABI_VERSION of include/linqt_gpu.h


def load():
    """Load liblinqt_gpu.so (raises if it is missing: build it with linqt_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("liblinqt_gpu.so is not built (run `python -m linqt_b200.build`); "
                               "linqt_b200 has no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.linqt_abi_version() != ABI_VERSION:
            raise RuntimeError("liblinqt_gpu.so has ABI version %d, the bindings expect %d: rebuild it"
                               % (L.linqt_abi_version(), ABI_VERSION))
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        msg = load().linqt_last_error()
        raise LinqtError(rc, msg.decode() if msg else "")
    return rc
