"""ctypes binding of the C ABI in include/seticore_b200.h (libseticore_b200.so).

The library is loaded from seticore_b200/_lib/ (built in-tree by seticore_b200.build).
There is no fallback: if the library is missing, loading raises.
"""
import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libseticore_b200.so")
# SETICORE_B200_LIBRARY overrides the path (e.g. to compare builds of the library).
LIB_PATH = os.environ.get("SETICORE_B200_LIBRARY", LIB_PATH)

SC_DD_OK = 0
SC_DD_EINVAL = 1
SC_DD_ECUDA = 2
SC_DD_ENOMEM = 3
SC_DD_ETRUNC = 4
SC_DD_EINTERNAL = 5
SC_DD_ESHAPE = 6
SC_DD_ELIMIT = 7
SC_DD_PRECISION_FP32 = 0
SC_DD_PRECISION_BF16 = 1
SC_DD_PRECISION_FP16 = 2
SC_DD_STATIC_MAX_CHANNELS = 1048576
NO_BEAM = -1

# Every symbol the header declares; tests check the library exports all of them.
EXPORTED = [
    "sc_dd_create", "sc_dd_destroy", "sc_dd_memory_usage", "sc_dd_rounded_timesteps",
    "sc_dd_search", "sc_dd_search_batch", "sc_dd_add_incoherent_power", "sc_dd_set_precision",
    "sc_dd_last_stats",
    "sc_dd_copy_channel_array", "sc_dd_last_error", "sc_dd_version", "sc_dd_search_static",
    "sc_dd_pool_create", "sc_dd_pool_destroy", "sc_dd_pool_configure", "sc_dd_pool_search",
    "sc_dd_pool_stats_get", "sc_dd_request_scratch_bytes", "sc_dd_pool_last_error",
    "sc_dd_prepare_coarse_channels", "sc_dd_gather_columns", "sc_dd_set_stage_wait_limit",
    "sc_dd_set_level_stripe_bytes",
    "sc_dd_set_exact_statistics",
    "sc_dd_set_paired_fp16",
]


class ScDdRequest(ctypes.Structure):
    _fields_ = [
        ("dev_input", ctypes.c_void_p),
        ("row_stride", ctypes.c_longlong),
        ("num_timesteps", ctypes.c_int),
        ("num_channels", ctypes.c_int),
        ("foff_mhz", ctypes.c_double),
        ("tsamp_s", ctypes.c_double),
        ("max_drift", ctypes.c_double),
        ("min_drift", ctypes.c_double),
        ("snr_threshold", ctypes.c_double),
        ("beam", ctypes.c_int),
        ("coarse_channel", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("pad", ctypes.c_int),
    ]


class ScDdPoolStats(ctypes.Structure):
    _fields_ = [
        ("calls", ctypes.c_longlong),
        ("sub_batches", ctypes.c_longlong),
        ("graph_replays", ctypes.c_longlong),
        ("graph_captures", ctypes.c_longlong),
        ("tuned_launches", ctypes.c_longlong),
        ("last_call_ms", ctypes.c_float),
        ("pad", ctypes.c_int),
    ]


class ScDdHit(ctypes.Structure):
    _fields_ = [
        ("index", ctypes.c_int),
        ("drift_steps", ctypes.c_int),
        ("drift_rate", ctypes.c_double),
        ("snr", ctypes.c_float),
        ("power", ctypes.c_float),
        ("incoherent_power", ctypes.c_float),
        ("coarse_channel", ctypes.c_int),
        ("beam", ctypes.c_int),
        ("num_timesteps", ctypes.c_int),
    ]


class ScDdStats(ctypes.Structure):
    _fields_ = [
        ("median", ctypes.c_float),
        ("std_dev", ctypes.c_float),
        ("mean", ctypes.c_float),
        ("threshold", ctypes.c_float),
        ("window_size", ctypes.c_int),
        ("min_drift_block", ctypes.c_int),
        ("max_drift_block", ctypes.c_int),
        ("num_candidates", ctypes.c_int),
        ("tree_ms", ctypes.c_float),
        ("search_ms", ctypes.c_float),
        ("precision", ctypes.c_int),
        ("recomputed_channels", ctypes.c_int),
        ("total_channels", ctypes.c_int),
        ("d2h_bytes", ctypes.c_int),
        ("norm_mean", ctypes.c_double),
        ("norm_std", ctypes.c_double),
        ("order_exact", ctypes.c_int),
        ("pad2", ctypes.c_int),
    ]


class DedopplerError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"seticore_b200 error {code}: {message}")
        self.code = code


_lib = None


def lib():
    """The loaded library (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} not found: build it with `python -m seticore_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        L.sc_dd_create.argtypes = [i, i, d, d, i, ctypes.POINTER(vp)]
        L.sc_dd_destroy.argtypes = [vp]
        L.sc_dd_memory_usage.argtypes = [vp]
        L.sc_dd_memory_usage.restype = ctypes.c_size_t
        L.sc_dd_rounded_timesteps.argtypes = [vp]
        L.sc_dd_search.argtypes = [vp, vp, ll, i, i, d, d, d, ctypes.POINTER(ScDdHit), i,
                                   ctypes.POINTER(i), vp]
        L.sc_dd_search_batch.argtypes = [vp, i, ctypes.POINTER(vp), ctypes.POINTER(ll), ctypes.POINTER(i),
                                         ctypes.POINTER(i), d, d, d, ctypes.POINTER(ScDdHit), i,
                                         ctypes.POINTER(i), vp]
        L.sc_dd_add_incoherent_power.argtypes = [vp, vp, ll, ctypes.POINTER(ScDdHit), i, vp]
        L.sc_dd_last_stats.argtypes = [vp, ctypes.POINTER(ScDdStats)]
        L.sc_dd_set_precision.argtypes = [vp, i]
        L.sc_dd_pool_create.argtypes = [ctypes.c_size_t, ctypes.POINTER(vp)]
        L.sc_dd_pool_destroy.argtypes = [vp]
        L.sc_dd_pool_configure.argtypes = [vp, i, i]
        L.sc_dd_pool_search.argtypes = [vp, ctypes.POINTER(ScDdRequest), i, ctypes.POINTER(ScDdHit), i,
                                        ctypes.POINTER(i), vp]
        L.sc_dd_pool_stats_get.argtypes = [vp, ctypes.POINTER(ScDdPoolStats)]
        L.sc_dd_request_scratch_bytes.argtypes = [ctypes.POINTER(ScDdRequest)]
        L.sc_dd_request_scratch_bytes.restype = ctypes.c_size_t
        L.sc_dd_pool_last_error.restype = ctypes.c_char_p
        L.sc_dd_search_static.argtypes = [vp, ll, i, i, d, d, i, i, d, d, d, ctypes.POINTER(ScDdHit), i,
                                          ctypes.POINTER(i), vp]
        L.sc_dd_copy_channel_array.argtypes = [vp, i, vp, vp]
        L.sc_dd_prepare_coarse_channels.argtypes = [vp, i, ll, ll, i, i, i, i, vp]
        L.sc_dd_gather_columns.argtypes = [vp, ll, i, i, vp, vp, i, vp, vp]
        L.sc_dd_set_stage_wait_limit.argtypes = [i]
        L.sc_dd_set_level_stripe_bytes.argtypes = [ctypes.c_longlong]
        L.sc_dd_set_exact_statistics.argtypes = [i]
        L.sc_dd_set_paired_fp16.argtypes = [i]
        L.sc_dd_last_error.restype = ctypes.c_char_p
        L.sc_dd_version.restype = ctypes.c_char_p
        for name in EXPORTED:
            getattr(L, name).restype = getattr(L, name).restype or ctypes.c_int
        L.sc_dd_last_error.restype = ctypes.c_char_p
        L.sc_dd_version.restype = ctypes.c_char_p
        L.sc_dd_memory_usage.restype = ctypes.c_size_t
        _lib = L
    return _lib


def check(rc, pool=False):
    if rc != SC_DD_OK:
        msg = (lib().sc_dd_pool_last_error() if pool else lib().sc_dd_last_error()).decode()
        raise DedopplerError(rc, msg)
    return rc
