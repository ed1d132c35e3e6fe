"""ctypes wrapper of the C oracle (oracle/liboracle.so). Test infrastructure only."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class Params(C.Structure):
    _fields_ = [
        ("n_replicas", C.c_int32),
        ("n_steps", C.c_int32),
        ("step_size", C.c_float),
        ("start_time", C.c_int64),
        ("window", C.c_int64),
        ("transition", C.c_int32),
        ("seed", C.c_uint64),
        ("exposed_duration", C.c_int32),
        ("infectious_duration", C.c_int32),
        ("resistant_duration", C.c_int32),
        ("infect_prob", C.c_float),
        ("initial_infected", C.c_float),
        ("initial_count", C.c_int32),
        ("beta", C.c_float),
        ("beta_per_replica", C.c_void_p),
        ("susceptibility", C.c_void_p),
        ("p_ei", C.c_float),
        ("p_ir", C.c_float),
        ("p_rs", C.c_float),
        ("has_exposed", C.c_int32),
        ("ir_to_s", C.c_int32),
        ("ncls_cap", C.c_int32),
        ("net_first", C.c_void_p),
        ("n_nets", C.c_int32),
        ("replica_offset", C.c_int32),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle oracle)")
        L = C.CDLL(path)
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_unit.argtypes = [C.c_uint32]
        L.orc_unit.restype = C.c_float
        L.orc_uniform.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_uniform.restype = C.c_float
        L.orc_infect_event.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float]
        L.orc_infect_event.restype = C.c_int
        L.orc_flow_event.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int]
        L.orc_flow_event.restype = C.c_int
        L.orc_threshold64.argtypes = [C.c_float, C.POINTER(C.c_int)]
        L.orc_threshold64.restype = C.c_uint64
        L.orc_one_minus_exp_neg.argtypes = [C.c_float]
        L.orc_one_minus_exp_neg.restype = C.c_float
        L.orc_timegm.argtypes = [C.c_int] * 6
        L.orc_timegm.restype = C.c_int64
        L.orc_parse_iso8601.argtypes = [C.c_char_p]
        L.orc_parse_iso8601.restype = C.c_int64
        L.orc_parse_file.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_store_coords.argtypes = [i64p, i64p, C.c_int64, i64p, i64p]
        L.orc_sort_order.argtypes = [i64p, i64p, C.c_int64, i64p]
        L.orc_nlists.argtypes = [i64p, i64p, C.c_int64]
        L.orc_nlists.restype = C.c_int64
        L.orc_window_hits.argtypes = [i64p, i64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, i64p]
        L.orc_window_hits.restype = C.c_int64
        L.orc_csr_f32.argtypes = [i64p, i64p, i32p, i32p, i64p, C.c_int64, C.c_int32, C.c_int64,
                                  C.c_int64, C.c_float, i32p, i32p, f32p]
        L.orc_csr_f32.restype = C.c_int64
        L.orc_csr_i32.argtypes = [i64p, i64p, i32p, i32p, i64p, C.c_int64, C.c_int32, C.c_int64,
                                  C.c_int64, i32p, i32p, i32p]
        L.orc_csr_i32.restype = C.c_int64
        L.orc_spmm_f32.argtypes = [i32p, i32p, f32p, C.c_int32, f32p, f32p, C.c_int32]
        L.orc_spmm_i64.argtypes = [i32p, i32p, i32p, C.c_int32, u8p, i64p, C.c_int32]
        L.orc_schedule.argtypes = [C.c_int64, C.c_float, C.c_int64, C.c_int32, i64p, i64p, f32p, i64p]
        L.orc_schedule.restype = C.c_int
        L.orc_run.argtypes = [i64p, i64p, i32p, i32p, C.c_int64, C.c_int32, C.POINTER(Params),
                              i32p, C.c_void_p]
        L.orc_run.restype = C.c_int
        L.orc_countdown_class.argtypes = [C.c_int32] * 4
        L.orc_countdown_class.restype = C.c_int
        _LIB = L
    return _LIB


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in ctr])
    k = (C.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [int(x) for x in o]


def uniform(seed, node, step, replica, stream=0):
    return lib().orc_uniform(seed, node, step, replica, stream)


def infect_event(seed, node, step, replica, P):
    """Geometric-mode infection decision of a replica (orc_infect_event)."""
    return bool(lib().orc_infect_event(seed, node, step, replica, float(P)))


def flow_event(seed, node, step, replica, p):
    """Flow decision (E->I, I->R, R->S) of a replica at per-step probability
    p (orc_threshold64 + orc_flow_event)."""
    always = C.c_int()
    T = lib().orc_threshold64(float(p), C.byref(always))
    return bool(lib().orc_flow_event(seed, node, step, replica, T, always.value))


def flow_threshold(p):
    """floor(p 2^64) for 0 < p < 1 (0 otherwise) and whether p >= 1."""
    always = C.c_int()
    T = lib().orc_threshold64(float(p), C.byref(always))
    return int(T), bool(always.value)


def one_minus_exp_neg(x):
    return lib().orc_one_minus_exp_neg(float(x))


def parse_file(path):
    """Returns dict(n_nodes, n_index, start, end, u, v, n_malformed) or raises."""
    L = lib()
    nn, ni, nc, nm = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
    ps, pe, pu, pv = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = L.orc_parse_file(path.encode(), C.byref(nn), C.byref(ni), C.byref(nc), C.byref(ps),
                          C.byref(pe), C.byref(pu), C.byref(pv), C.byref(nm))
    if rc != 0:
        return {"error": rc, "n_nodes": nn.value}
    n = nc.value

    def take(p, ctype, dtype):
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), shape=(n,)).astype(dtype).copy()
        L.orc_free(p)
        return arr

    return {
        "error": 0,
        "n_nodes": nn.value,
        "n_index": ni.value,
        "start": take(ps, C.c_int64, np.int64),
        "end": take(pe, C.c_int64, np.int64),
        "u": take(pu, C.c_int32, np.int32),
        "v": take(pv, C.c_int32, np.int32),
        "n_malformed": nm.value,
    }


def store_coords(start, end):
    start = np.ascontiguousarray(start, np.int64)
    end = np.ascontiguousarray(end, np.int64)
    os_, oe = np.zeros_like(start), np.zeros_like(end)
    lib().orc_store_coords(start, end, len(start), os_, oe)
    return os_, oe


def sorted_index(start, end, u, v):
    """Stored coordinates in sorted order: (s, e, u, v, perm, nlists)."""
    s2, e2 = store_coords(start, end)
    perm = sort_order(s2, e2)
    ss, se = s2[perm].copy(), e2[perm].copy()
    return ss, se, np.asarray(u, np.int32)[perm].copy(), np.asarray(v, np.int32)[perm].copy(), perm, nlists(ss, se)


def hit_coords(s, e, ws):
    """Coordinates a stored hit (s, e) is handed to the CSR builder with."""
    hs, he = C.c_int64(), C.c_int64()
    lib().orc_hit_coords(C.c_int64(int(s)), C.c_int64(int(e)), C.c_int64(int(ws)), C.byref(hs), C.byref(he))
    return hs.value, he.value


def sort_order(start, end):
    start = np.ascontiguousarray(start, np.int64)
    end = np.ascontiguousarray(end, np.int64)
    perm = np.zeros(len(start), np.int64)
    lib().orc_sort_order(start, end, len(start), perm)
    return perm


def nlists(s_start, s_end):
    return lib().orc_nlists(np.ascontiguousarray(s_start, np.int64), np.ascontiguousarray(s_end, np.int64),
                            len(s_start))


def window_hits(s_start, s_end, nl, ws, we):
    out = np.zeros(max(len(s_start), 1), np.int64)
    k = lib().orc_window_hits(np.ascontiguousarray(s_start, np.int64), np.ascontiguousarray(s_end, np.int64),
                              len(s_start), nl, ws, we, out)
    return out[:k]


def csr_f32(ss, se, su, sv, hits, n_nodes, ws, we, scale):
    hits = np.ascontiguousarray(hits, np.int64)
    rp = np.zeros(n_nodes + 1, np.int32)
    col = np.zeros(max(2 * len(hits), 1), np.int32)
    val = np.zeros(max(2 * len(hits), 1), np.float32)
    nnz = lib().orc_csr_f32(ss, se, su, sv, hits, len(hits), n_nodes, ws, we, scale, rp, col, val)
    return rp, col[:nnz], val[:nnz]


def csr_i32(ss, se, su, sv, hits, n_nodes, ws, we):
    hits = np.ascontiguousarray(hits, np.int64)
    rp = np.zeros(n_nodes + 1, np.int32)
    col = np.zeros(max(2 * len(hits), 1), np.int32)
    val = np.zeros(max(2 * len(hits), 1), np.int32)
    nnz = lib().orc_csr_i32(ss, se, su, sv, hits, len(hits), n_nodes, ws, we, rp, col, val)
    return rp, col[:nnz], val[:nnz]


def spmm_f32(rp, col, val, n, b_colmajor, m):
    c = np.zeros(n * m, np.float32)
    lib().orc_spmm_f32(np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(col, np.int32),
                       np.ascontiguousarray(val, np.float32), n,
                       np.ascontiguousarray(b_colmajor, np.float32), c, m)
    return c


def spmm_i64(rp, col, val, n, b_colmajor, m):
    c = np.zeros(n * m, np.int64)
    lib().orc_spmm_i64(np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(col, np.int32),
                       np.ascontiguousarray(val, np.int32), n,
                       np.ascontiguousarray(b_colmajor, np.uint8), c, m)
    return c


def schedule(start_time, step_size, window, n_steps):
    ws = np.zeros(max(n_steps, 1), np.int64)
    we = np.zeros(max(n_steps, 1), np.int64)
    sc = np.zeros(max(n_steps, 1), np.float32)
    ts = np.zeros(max(n_steps, 1), np.int64)
    rc = lib().orc_schedule(start_time, step_size, window, n_steps, ws, we, sc, ts)
    if rc:
        raise ValueError("schedule overflow")
    return ws[:n_steps], we[:n_steps], sc[:n_steps], ts[:n_steps]


def run(start, end, u, v, n_nodes, node_states=False, **kw):
    """Full replay on the CPU.  Returns counts (T+1, M, 4) [and node states]."""
    p = Params()
    defaults = dict(n_replicas=1000, n_steps=42, step_size=3600.0, start_time=946713600, window=3600,
                    transition=0, seed=1, exposed_duration=0, infectious_duration=0, resistant_duration=0,
                    infect_prob=0.0, initial_infected=0.0, initial_count=0, beta=0.0, p_ei=0.0, p_ir=0.0,
                    p_rs=0.0, has_exposed=1, ir_to_s=0, ncls_cap=1)
    keep = []
    for k, val in {**defaults, **kw}.items():
        if k in ("beta_per_replica", "susceptibility", "net_first"):
            continue
        setattr(p, k, val)
    for k in ("beta_per_replica", "susceptibility"):
        if kw.get(k) is not None:
            arr = np.ascontiguousarray(kw[k], np.float32)
            keep.append(arr)
            setattr(p, k, arr.ctypes.data)
    n_nets = 1
    if kw.get("net_first") is not None:
        nf = np.ascontiguousarray(kw["net_first"], np.int32)
        keep.append(nf)
        n_nets = len(nf) - 1
        p.net_first, p.n_nets = nf.ctypes.data, n_nets
    T, M = p.n_steps, p.n_replicas
    counts = np.zeros((T + 1) * n_nets * M * 4, np.int32)
    ns = np.zeros((T + 1) * M * n_nodes, np.uint8) if node_states else None
    rc = lib().orc_run(np.ascontiguousarray(start, np.int64), np.ascontiguousarray(end, np.int64),
                       np.ascontiguousarray(u, np.int32), np.ascontiguousarray(v, np.int32), len(start),
                       n_nodes, C.byref(p), counts, ns.ctypes.data if ns is not None else None)
    if rc:
        raise RuntimeError(f"orc_run failed ({rc})")
    counts = counts.reshape(T + 1, n_nets, M, 4) if n_nets > 1 or kw.get("net_first") is not None \
        else counts.reshape(T + 1, M, 4)
    if node_states:
        return counts, ns.reshape(T + 1, M, n_nodes)
    return counts
