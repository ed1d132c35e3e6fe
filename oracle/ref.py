"""ctypes wrapper of the reference built from its own sources (oracle/_ref).

Test infrastructure only: used to pin the C oracle and to generate the golden
fixtures under tests/golden/.  Built by `make -C oracle ref` where the
reference tree is present.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
REPLAY_REF = os.path.join(REF_DIR, "replay_ref")
CONTACT_NETWORK_REF = os.path.join(REF_DIR, "contact_network_ref")
_LIB = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def available():
    return os.path.exists(os.path.join(REF_DIR, "libref_shim.so"))


def lib():
    global _LIB
    if _LIB is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_shim.so"))
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_parse.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p),
                                C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.ref_parse.restype = C.c_int
        L.ref_window_query.argtypes = [i64p, i64p, i32p, i32p, C.c_int, C.c_int64, C.c_int64,
                                       C.POINTER(C.c_int), C.POINTER(C.c_int), i64p, i64p, i32p, i32p]
        L.ref_window_query.restype = C.c_int
        L.ref_build_csr.argtypes = [i64p, i64p, i32p, i32p, C.c_int, C.c_int, C.c_int64, C.c_int64,
                                    C.c_float, i32p, i32p, f32p]
        L.ref_build_csr.restype = C.c_long
        L.ref_cpu_spmm.argtypes = [i32p, i32p, f32p, C.c_long, C.c_int, f32p, f32p, C.c_int]
        L.ref_set_durations.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float]
        L.ref_infectious.argtypes = [i32p, f32p, C.c_int, C.c_int]
        L.ref_infection_prob.argtypes = [f32p, i32p, C.c_int, C.c_int, C.c_float]
        L.ref_update_countdown.argtypes = [i32p, C.c_int, C.c_int, C.c_float]
        L.ref_write_state.argtypes = [C.c_char_p, C.c_char_p, i32p, C.c_int, C.c_int, C.c_int64]
        L.ref_write_state.restype = C.c_int
        _LIB = L
    return _LIB


def parse(path, quiet=True):
    L = lib()
    nn = C.c_int()
    ps, pe, pu, pv = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    n = L.ref_parse(path.encode(), 1 if quiet else 0, C.byref(nn), C.byref(ps), C.byref(pe), C.byref(pu),
                    C.byref(pv))
    if n < 0:
        return {"error": 1, "n_nodes": nn.value}

    def take(p, ctype, dtype):
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), shape=(max(n, 1),))[:n].astype(dtype).copy()
        L.ref_free(p)
        return arr

    return {"error": 0, "n_nodes": nn.value, "start": take(ps, C.c_int64, np.int64),
            "end": take(pe, C.c_int64, np.int64), "u": take(pu, C.c_int32, np.int32),
            "v": take(pv, C.c_int32, np.int32)}


def window_query(start, end, u, v, ws, we):
    n = len(start)
    hs, he = np.zeros(max(n, 1), np.int64), np.zeros(max(n, 1), np.int64)
    hu, hv = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.int32)
    nl, nc = C.c_int(), C.c_int()
    k = lib().ref_window_query(np.ascontiguousarray(start, np.int64), np.ascontiguousarray(end, np.int64),
                               np.ascontiguousarray(u, np.int32), np.ascontiguousarray(v, np.int32), n, ws, we,
                               C.byref(nl), C.byref(nc), hs, he, hu, hv)
    return {"nlists": nl.value, "n_compact": nc.value, "start": hs[:k], "end": he[:k], "u": hu[:k], "v": hv[:k]}


def build_csr(hs, he, hu, hv, n_nodes, ws, we, scale):
    k = len(hs)
    rp = np.zeros(n_nodes + 1, np.int32)
    col = np.zeros(max(2 * k, 1), np.int32)
    val = np.zeros(max(2 * k, 1), np.float32)
    nnz = lib().ref_build_csr(np.ascontiguousarray(hs, np.int64), np.ascontiguousarray(he, np.int64),
                              np.ascontiguousarray(hu, np.int32), np.ascontiguousarray(hv, np.int32), k, n_nodes,
                              ws, we, scale, rp, col, val)
    return rp, col[:nnz], val[:nnz]


def cpu_spmm(rp, col, val, n, b, m):
    c = np.zeros(n * m, np.float32)
    lib().ref_cpu_spmm(np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(col, np.int32),
                       np.ascontiguousarray(val, np.float32), len(col), n, np.ascontiguousarray(b, np.float32), c, m)
    return c


def run_cli(args, timeout=600):
    """Runs the reference executable; returns CompletedProcess."""
    return subprocess.run([REPLAY_REF] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
