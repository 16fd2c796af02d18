"""Python bindings of the oracles.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() (to check its result) and bench.py's CPU-baseline /
reference legs use this module; the product (seticore_b200/) never imports it.

  Oracle("port")       -- oracle/_build/liboracle.so: CPU restatement of the reference
  Oracle("reference")  -- oracle/_ref/libref_cpu.so: the same host driver with every tree
                          step done by the reference's own taylorOneStepOneChannel
  RefGpu               -- oracle/_ref/libref_gpu.so: the reference's own GPU Dedopplerer
                          (dedoppler.cu, taylor.cu, ...) built for sm_100a
Build them with `make -C oracle` (needs the reference tree for the _ref libraries).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATHS = {
    "port": os.path.join(HERE, "_build", "liboracle.so"),
    "reference": os.path.join(HERE, "_ref", "libref_cpu.so"),
    "reference_gpu": os.path.join(HERE, "_ref", "libref_gpu.so"),
}

_f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OracleHit(ctypes.Structure):
    _fields_ = [("index", ctypes.c_int), ("drift_steps", ctypes.c_int),
                ("drift_rate", ctypes.c_double), ("snr", ctypes.c_float), ("power", ctypes.c_float)]


class OracleStats(ctypes.Structure):
    _fields_ = [("median", ctypes.c_float), ("std_dev", ctypes.c_float), ("mean", ctypes.c_float),
                ("threshold", ctypes.c_float), ("window_size", ctypes.c_int),
                ("min_drift_block", ctypes.c_int), ("max_drift_block", ctypes.c_int),
                ("drift_rate_resolution", ctypes.c_double)]


class RefHit(ctypes.Structure):
    _fields_ = [("index", ctypes.c_int), ("drift_steps", ctypes.c_int), ("drift_rate", ctypes.c_double),
                ("snr", ctypes.c_float), ("power", ctypes.c_float), ("incoherent_power", ctypes.c_float),
                ("coarse_channel", ctypes.c_int), ("beam", ctypes.c_int), ("num_timesteps", ctypes.c_int),
                ("frequency", ctypes.c_double)]


class RefEventHit(ctypes.Structure):
    _fields_ = [("present", ctypes.c_int), ("index", ctypes.c_int), ("drift_steps", ctypes.c_int),
                ("snr", ctypes.c_float), ("power", ctypes.c_float)]


def available(kind="port"):
    return os.path.exists(PATHS[kind])


class Oracle:
    def __init__(self, kind="port"):
        path = PATHS[kind]
        if not os.path.exists(path):
            raise OSError(f"{path} missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.oracle_taylor_f32.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32]
        L.oracle_taylor_f64.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64]
        L.oracle_path_sum.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_path_sum.restype = ctypes.c_float
        L.oracle_incoherent_power.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_incoherent_power.restype = ctypes.c_float
        L.oracle_search.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.POINTER(OracleHit), ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.POINTER(OracleStats)]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        self.lib = L
        self.kind = kind

    def set_threads(self, n):
        self.lib.oracle_set_threads(int(n))

    def max_threads(self):
        return int(self.lib.oracle_max_threads())

    def taylor(self, x, db):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty_like(x)
        self.lib.oracle_taylor_f32(x, x.shape[0], x.shape[1], int(db), out)
        return out

    def taylor_f64(self, x, db):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty(x.shape, dtype=np.float64)
        self.lib.oracle_taylor_f64(x, x.shape[0], x.shape[1], int(db), out)
        return out

    def path_sum(self, x, db, off, c):
        x = np.ascontiguousarray(x, dtype=np.float32)
        return float(self.lib.oracle_path_sum(x, x.shape[0], x.shape[1], db, off, c))

    def incoherent_power(self, x, drift_steps, index):
        x = np.ascontiguousarray(x, dtype=np.float32)
        return float(self.lib.oracle_incoherent_power(x, x.shape[0], x.shape[1], drift_steps, index))

    def search(self, x, foff_mhz, tsamp, max_drift, min_drift, snr_threshold, arrays=False):
        """Returns (hits as list of dicts, stats dict[, arrays dict])."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        Tr, N = x.shape
        cap = max(16, N // 2 + 2)
        hits = (OracleHit * cap)()
        st = OracleStats()
        top = np.zeros(N, np.float32)
        tdb = np.zeros(N, np.int32)
        toff = np.zeros(N, np.int32)
        cs = np.zeros(N, np.float32)
        n = self.lib.oracle_search(x, Tr, N, foff_mhz, tsamp, max_drift, min_drift, snr_threshold, hits, cap,
                                   top.ctypes.data, tdb.ctypes.data, toff.ctypes.data, cs.ctypes.data,
                                   ctypes.byref(st))
        if n < 0:
            raise ValueError("oracle: window size < 1 for this max_drift")
        out = [dict(index=h.index, drift_steps=h.drift_steps, drift_rate=h.drift_rate, snr=h.snr, power=h.power)
               for h in hits[:n]]
        stats = {k: getattr(st, k) for k, _ in OracleStats._fields_}
        if arrays:
            return out, stats, dict(top=top, top_db=tdb, top_off=toff, colsum=cs)
        return out, stats


class RefGpu:
    """The reference's own GPU Dedopplerer (built for sm_100a).  Needs a GPU."""

    def __init__(self):
        path = PATHS["reference_gpu"]
        if not os.path.exists(path):
            raise OSError(f"{path} missing: run `make -C oracle` where the reference tree exists")
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.ref_gpu_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.ref_gpu_create.restype = vp
        L.ref_gpu_destroy.argtypes = [vp]
        L.ref_gpu_load.argtypes = [vp, _f32]
        L.ref_gpu_search.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.POINTER(RefHit), ctypes.c_int]
        L.ref_gpu_time_search.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ref_gpu_time_search.restype = ctypes.c_double
        L.ref_gpu_add_incoherent.argtypes = [vp, ctypes.POINTER(RefHit), ctypes.c_int]
        L.ref_gpu_taylor.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32]
        if hasattr(L, "ref_find_events"):
            L.ref_find_events.argtypes = [
                ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                ctypes.POINTER(ctypes.POINTER(ctypes.c_float)), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                ctypes.c_double, ctypes.c_double, ctypes.POINTER(RefEventHit), ctypes.c_int]
            L.ref_find_events.restype = ctypes.c_int
        self.lib = L

    def find_events(self, files, max_drift, snr_on, snr_off, cap=1024):
        """The reference's findEvents (find_events.cpp:65-226) over in-memory files.

        files: dicts with `rows` ([num_timesteps][num_coarse * coarse_size] float32),
        source_name, tstart and the shared shape/metadata keys coarse_size, num_coarse, fch1,
        foff, tsamp, has_dc_spike.  Returns the events as lists with one entry per file:
        None or a dict of the hit's index, drift_steps, snr and power."""
        if not hasattr(self.lib, "ref_find_events"):
            raise OSError("libref_gpu.so predates ref_find_events: rebuild with `make -C oracle`")
        n = len(files)
        f0 = files[0]
        rows = [np.ascontiguousarray(f["rows"], dtype=np.float32) for f in files]
        names = (ctypes.c_char_p * n)(*[f["source_name"].encode() for f in files])
        tstarts = (ctypes.c_double * n)(*[float(f["tstart"]) for f in files])
        ptrs = (ctypes.POINTER(ctypes.c_float) * n)(
            *[r.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) for r in rows])
        out = (RefEventHit * (cap * n))()
        ne = self.lib.ref_find_events(n, names, tstarts, ptrs, rows[0].shape[0], int(f0["coarse_size"]),
                                      int(f0["num_coarse"]), float(f0["fch1"]), float(f0["foff"]),
                                      float(f0["tsamp"]), int(bool(f0["has_dc_spike"])), float(max_drift),
                                      float(snr_on), float(snr_off), out, cap)
        if ne < 0:
            raise RuntimeError("reference findEvents raised")
        events = []
        for e in range(min(ne, cap)):
            ev = []
            for k in range(n):
                h = out[e * n + k]
                ev.append(dict(index=h.index, drift_steps=h.drift_steps, snr=h.snr, power=h.power)
                          if h.present else None)
            events.append(ev)
        return events

    def taylor(self, x, db):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty_like(x)
        rc = self.lib.ref_gpu_taylor(x, x.shape[0], x.shape[1], int(db), out)
        assert rc == 0, rc
        return out

    class Ctx:
        def __init__(self, ref, T, N, foff_mhz, tsamp):
            self.ref = ref
            self.h = ref.lib.ref_gpu_create(T, N, foff_mhz, tsamp)

        def load(self, x):
            self.ref.lib.ref_gpu_load(self.h, np.ascontiguousarray(x, dtype=np.float32))

        def search(self, beam, coarse, max_drift, min_drift, snr):
            cap = 65536
            hits = (RefHit * cap)()
            n = self.ref.lib.ref_gpu_search(self.h, beam, coarse, max_drift, min_drift, snr, hits, cap)
            return [dict(index=h.index, drift_steps=h.drift_steps, drift_rate=h.drift_rate, snr=h.snr,
                         power=h.power, beam=h.beam, coarse_channel=h.coarse_channel) for h in hits[:n]]

        def time_search(self, max_drift, min_drift, snr, iters):
            return float(self.ref.lib.ref_gpu_time_search(self.h, max_drift, min_drift, snr, iters))

        def add_incoherent(self, hits):
            arr = (RefHit * len(hits))()
            for i, h in enumerate(hits):
                arr[i].index = h["index"]
                arr[i].drift_steps = h["drift_steps"]
                arr[i].drift_rate = h.get("drift_rate", 0.0)
                arr[i].snr = h.get("snr", 0.0)
                arr[i].power = h.get("power", 0.0)
                arr[i].beam = -1
                arr[i].num_timesteps = 16
            self.ref.lib.ref_gpu_add_incoherent(self.h, arr, len(hits))
            return [dict(index=a.index, drift_steps=a.drift_steps, incoherent_power=a.incoherent_power)
                    for a in arr]

        def close(self):
            if self.h:
                self.ref.lib.ref_gpu_destroy(self.h)
                self.h = None

    def context(self, T, N, foff_mhz, tsamp):
        return RefGpu.Ctx(self, T, N, foff_mhz, tsamp)
