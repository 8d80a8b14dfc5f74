"""ctypes mirror of include/sparc_gpu.h (structs, status codes, loader).

The structures here must match the C header field for field; the CPU test
suite checks their sizes against the compiled library's view of them.
"""
import ctypes as C
import os

SPARC_OK = 0
SPARC_ERR_INVALID = -1
SPARC_ERR_CUDA = -2
SPARC_ERR_NOMEM = -3
SPARC_ERR_UNSTABLE = -4
SPARC_ERR_ORDER = -5
SPARC_ERR_TIMEOUT = -6
SPARC_ERR_NODEVICE = -7

ERR_NAMES = {
    SPARC_ERR_INVALID: "SPARC_ERR_INVALID",
    SPARC_ERR_CUDA: "SPARC_ERR_CUDA",
    SPARC_ERR_NOMEM: "SPARC_ERR_NOMEM",
    SPARC_ERR_UNSTABLE: "SPARC_ERR_UNSTABLE",
    SPARC_ERR_ORDER: "SPARC_ERR_ORDER",
    SPARC_ERR_TIMEOUT: "SPARC_ERR_TIMEOUT",
    SPARC_ERR_NODEVICE: "SPARC_ERR_NODEVICE",
}

SPARC_FP64 = 0
SPARC_FP32 = 1

SPARC_REQ_QUEUED = 0
SPARC_REQ_ADMITTED = 1
SPARC_REQ_RUNNING = 2
SPARC_REQ_DONE = 3
SPARC_REQ_FAILED = 4
SPARC_REQ_COLLECTED = 5

SPARC_SRC_NONE = 0
SPARC_SRC_PULSE = 1
SPARC_SRC_PSR = 2
SPARC_SRC_RANDOM = 3


class SparcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("magnetic", C.c_int32), ("periodic", C.c_int32),
        ("use_pml", C.c_int32), ("use_hpml", C.c_int32),
        ("stabilise", C.c_int32),
        ("filter_mode_xy", C.c_int32), ("filter_mode_z", C.c_int32),
        ("block_x", C.c_int32), ("block_y", C.c_int32), ("block_z", C.c_int32),
        ("npml_xb", C.c_int32), ("npml_xt", C.c_int32),
        ("npml_yb", C.c_int32), ("npml_yt", C.c_int32),
        ("npml_zb", C.c_int32), ("npml_zt", C.c_int32),
        ("pml_xb", C.c_double * 4), ("pml_xt", C.c_double * 4),
        ("pml_yb", C.c_double * 4), ("pml_yt", C.c_double * 4),
        ("pml_zb", C.c_double * 4), ("pml_zt", C.c_double * 4),
        ("xlength", C.c_double), ("ylength", C.c_double),
        ("timestep", C.c_double),
        ("s_xy", C.c_double), ("s_z", C.c_double),
        ("t_xy", C.c_double), ("t_z", C.c_double),
        ("maxva", C.c_double),
        ("sp_str", C.c_double), ("sp_length", C.c_double),
        ("sp_decay", C.c_double),
        ("precision", C.c_int32),
        ("damping", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]


class SparcPulse(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("px", "py", "pz", "sr", "sz", "amp", "t0", "t1")]


class SparcSource(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("dir", C.c_int32), ("init", C.c_int64),
        ("amp", C.c_double), ("t0", C.c_double), ("t1", C.c_double),
        ("st", C.c_double), ("px", C.c_double), ("py", C.c_double),
        ("pz", C.c_double), ("sr", C.c_double), ("sz", C.c_double),
        ("psr_st", C.c_double),
        ("npulses", C.c_int32), ("pad", C.c_int32),
        ("pulses", C.POINTER(SparcPulse)),
        ("cadforcing", C.c_double), ("rnd_ampl", C.c_double),
        ("rnd_depth", C.c_double), ("rnd_sigma", C.c_double),
        ("nseries", C.c_int32), ("pad2", C.c_int32),
        ("series", C.POINTER(C.c_double)),
    ]


class SparcDiag(C.Structure):
    _fields_ = [
        ("ke_norm", C.c_double), ("min_rho", C.c_double),
        ("min_p", C.c_double), ("iteration", C.c_int64),
        ("fail_iteration", C.c_int64),
    ]


class SparcTrol(C.Structure):
    """include/sparc_trol.h: a .trol parameter file as read by
    sparc_read_trol (READ_SPARC_PARAMETERS, initialize.f90:1385-1924)."""
    _fields_ = [
        ("params", SparcParams), ("source", SparcSource),
        ("pulse", C.c_int32), ("psr_npulses", C.c_int32),
        ("restart", C.c_int32), ("time0", C.c_int32),
        ("twod", C.c_int32), ("twop5d", C.c_int32), ("displ", C.c_int32),
        ("flows", C.c_int32), ("damping", C.c_int32),
        ("timestamp_size", C.c_int32),
        ("xcb", C.c_int32), ("xct", C.c_int32), ("ycb", C.c_int32),
        ("yct", C.c_int32), ("zcb", C.c_int32), ("zct", C.c_int32),
        ("fullout", C.c_int32), ("chunkout", C.c_int32),
        ("solartime", C.c_double), ("wall_time", C.c_double),
        ("fulloutputcad", C.c_double), ("chunkoutputcad", C.c_double),
        ("minsavtime", C.c_double),
        ("maxtime", C.c_int64), ("init", C.c_int64),
        ("xyfreq", C.c_int64), ("zfreq", C.c_int64),
        ("fulloutputsteps", C.c_int64), ("chunkoutputsteps", C.c_int64),
        ("num_steps", C.c_int64),
        ("lines_read", C.c_int32), ("stopped_line", C.c_int32),
        ("dir_bkg", C.c_char * 200), ("dir_out", C.c_char * 200),
        ("simname", C.c_char * 240), ("forcingfunc", C.c_char * 200),
    ]


class SparcError(RuntimeError):
    """A negative status returned across the C ABI."""

    def __init__(self, code, where, detail=""):
        self.code = code
        name = ERR_NAMES.get(code, str(code))
        msg = f"{where} failed with {name}"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "_lib", "libsparc_gpu.so")

# Every entry point declared in include/sparc_gpu.h and include/sparc_trol.h.
EXPORTS = [
    "sparc_create", "sparc_destroy", "sparc_set_background",
    "sparc_set_source", "sparc_sizes", "sparc_set_state", "sparc_get_state",
    "sparc_step", "sparc_filter_vars", "sparc_run", "sparc_set_zchunk",
    "sparc_get_zchunk", "sparc_tune", "sparc_diagnostics",
    "sparc_synchronize", "sparc_stream", "sparc_launch_count",
    "sparc_derivative", "sparc_filter_field", "sparc_get_coeff",
    "sparc_get_scalars", "sparc_last_error",
    "sparc_batch_create", "sparc_batch_destroy", "sparc_batch_add",
    "sparc_batch_remove", "sparc_batch_run", "sparc_batch_remaining",
    "sparc_batch_set_tiles", "sparc_batch_get_tiles",
    "sparc_batch_synchronize", "sparc_batch_stream",
    "sparc_batch_launch_count", "sparc_batch_last_error",
    "sparc_batch_tune", "sparc_ke_norm_noalloc", "sparc_inject_wait_timeout",
    "sparc_estimate_bytes", "sparc_server_create", "sparc_server_destroy",
    "sparc_serve_submit", "sparc_serve_next", "sparc_serve_params",
    "sparc_serve_attach", "sparc_serve_result", "sparc_serve_release",
    "sparc_serve_state", "sparc_serve_stats", "sparc_server_last_error",
    "sparc_read_trol", "sparc_parse_trol",
]

_lib = None


def _declare(lib):
    P = C.POINTER
    d = C.POINTER(C.c_double)
    h = C.c_void_p
    sig = {
        "sparc_create": (C.c_int, [P(SparcParams), C.c_int, P(C.c_void_p)]),
        "sparc_read_trol": (C.c_int, [C.c_char_p, P(SparcTrol), C.c_char_p, C.c_int]),
        "sparc_parse_trol": (C.c_int, [C.c_char_p, P(SparcTrol), C.c_char_p, C.c_int]),
        "sparc_destroy": (C.c_int, [h]),
        "sparc_set_background": (C.c_int, [h, d, d, d, d, d, d, d, d]),
        "sparc_set_source": (C.c_int, [h, P(SparcSource)]),
        "sparc_sizes": (C.c_int, [h, P(C.c_int64), P(C.c_int64)]),
        "sparc_set_state": (C.c_int, [h, d, d]),
        "sparc_get_state": (C.c_int, [h, d, d]),
        "sparc_step": (C.c_int, [h, C.c_int64]),
        "sparc_filter_vars": (C.c_int, [h, C.c_int64]),
        "sparc_run": (C.c_int, [h, C.c_int64, C.c_int64]),
        "sparc_set_zchunk": (C.c_int, [h, C.c_int]),
        "sparc_get_zchunk": (C.c_int, [h, P(C.c_int)]),
        "sparc_tune": (C.c_int, [h, C.c_int64, C.c_int, P(C.c_int64), P(C.c_int)]),
        "sparc_diagnostics": (C.c_int, [h, P(SparcDiag)]),
        "sparc_synchronize": (C.c_int, [h]),
        "sparc_stream": (C.c_int, [h, P(C.c_void_p)]),
        "sparc_launch_count": (C.c_int, [h, P(C.c_int64)]),
        "sparc_derivative": (C.c_int, [h, C.c_int, C.c_int, d, d]),
        "sparc_filter_field": (C.c_int, [h, C.c_int, d, d]),
        "sparc_get_coeff": (C.c_int, [h, C.c_char_p, d, P(C.c_int64)]),
        "sparc_get_scalars": (C.c_int, [h, d]),
        "sparc_last_error": (C.c_char_p, [h]),
        "sparc_batch_create": (C.c_int, [C.c_int, C.c_int, P(C.c_void_p)]),
        "sparc_batch_destroy": (C.c_int, [h]),
        "sparc_batch_add": (C.c_int, [h, h, C.c_int64, C.c_int64,
                                      P(C.c_int)]),
        "sparc_batch_remove": (C.c_int, [h, C.c_int]),
        "sparc_batch_run": (C.c_int, [h, C.c_int64]),
        "sparc_batch_remaining": (C.c_int, [h, P(C.c_int64)]),
        "sparc_batch_set_tiles": (C.c_int, [h, C.c_int, C.c_int]),
        "sparc_batch_get_tiles": (C.c_int, [h, P(C.c_int), P(C.c_int)]),
        "sparc_batch_synchronize": (C.c_int, [h]),
        "sparc_batch_stream": (C.c_int, [h, P(C.c_void_p)]),
        "sparc_batch_launch_count": (C.c_int, [h, P(C.c_int64)]),
        "sparc_batch_last_error": (C.c_char_p, [h]),
        "sparc_batch_tune": (C.c_int, [h, C.c_int, P(C.c_int), P(C.c_int)]),
        "sparc_ke_norm_noalloc": (C.c_int, [h, d]),
        "sparc_inject_wait_timeout": (C.c_int, [h, C.c_int64]),
        "sparc_estimate_bytes": (C.c_int, [P(SparcParams), P(C.c_int64),
                                           P(C.c_int64)]),
        "sparc_server_create": (C.c_int, [C.c_int, C.c_int, C.c_int64,
                                          C.c_int, P(C.c_void_p)]),
        "sparc_server_destroy": (C.c_int, [h]),
        "sparc_serve_submit": (C.c_int, [h, P(SparcParams), C.c_int64,
                                         C.c_int64, P(C.c_int64)]),
        "sparc_serve_next": (C.c_int, [h, C.c_int, C.c_int64, P(C.c_int64)]),
        "sparc_serve_params": (C.c_int, [h, C.c_int64, P(SparcParams),
                                         P(C.c_int64), P(C.c_int64)]),
        "sparc_serve_attach": (C.c_int, [h, C.c_int64, h]),
        "sparc_serve_result": (C.c_int, [h, C.c_int64, P(C.c_void_p), d,
                                         P(C.c_int)]),
        "sparc_serve_release": (C.c_int, [h, C.c_int64]),
        "sparc_serve_state": (C.c_int, [h, C.c_int64, P(C.c_int)]),
        "sparc_serve_stats": (C.c_int, [h, d]),
        "sparc_server_last_error": (C.c_char_p, [h]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def load(path=None):
    """Load libsparc_gpu.so (built in-tree by sparc2_b200.build).

    Raises FileNotFoundError when the library has not been built: there is
    no fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    # SPARC_GPU_LIB: another build of the same library (A/B timing)
    p = path or os.environ.get("SPARC_GPU_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(
            f"{p} is missing; build it with `python -c 'import "
            f"sparc2_b200.build as b; b.build()'`")
    lib = _declare(C.CDLL(p))
    if path is None:
        _lib = lib
    return lib


def dptr(arr):
    """double* of a C-contiguous float64 numpy array (or NULL for None)."""
    if arr is None:
        return C.cast(None, C.POINTER(C.c_double))
    assert arr.dtype.name == "float64" and arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(C.c_double))
