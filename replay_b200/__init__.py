"""replay_b200: Monte Carlo SEIR replay over temporal contact networks on B200.

Python mirror of the `replay` command line (the reference's only interface,
tool/gpu_cpu_temporal_sim.cu:570-699) over the libreplay C ABI:

    g = Graph.load("contacts.txt")              # NODE_LIST + `u, v, t0, t1;` lines
    sim = Simulation(g, M=1000, iterations=168, step_size=3600,
                     initial_infected=0.01, infect_prob=0.0695,
                     exposed_duration=172800, infectious_duration=432000)
    counts = sim.run()                           # (iterations+1, M, 4) int32
    # columns: exposed, infectious, resistant, susceptible (summary CSV order)

Keyword names follow the CLI flags (--M, --iterations, --step-size,
--initial-infected, --infect-prob, --exposed-duration, ...); the additive
geometric mode takes transition="geometric", beta, p_ei, p_ir, p_rs.
Every simulation runs on the GPU; there is no CPU fallback.
"""
import ctypes as C
import weakref

import numpy as np

from . import _lib
from ._lib import CLI_PATH, ReplayError, check, lib

__all__ = ["Graph", "Simulation", "ReplayError", "window_csr", "parse_contacts", "batch_networks", "CLI_PATH",
           "version", "release_cached_memory"]


def version():
    return lib().rp_version().decode()


def release_cached_memory():
    """Returns the device blocks kept from closed graphs and simulations
    (closing a handle keeps its blocks, up to 8 GiB per device, for the
    next one) to the driver."""
    lib().rp_release_cached_memory()


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def parse_contacts(path):
    """Parses a contact file on the host (no GPU work).

    Returns dict(n_nodes, n_index, n_malformed, start, end, u, v): int64
    Unix-second intervals and int32 compressed node indices (u <= v, order of
    first appearance), in file order.  Raises ReplayError where the reference
    parser fails (unreadable file, bad NODE_LIST header, no contacts).
    """
    L = lib()
    nn, ni = C.c_int32(), C.c_int32()
    nc, nm = C.c_int64(), C.c_int64()
    ps, pe, pu, pv = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(L.rp_parse_contacts(str(path).encode(), C.byref(nn), C.byref(ni), C.byref(nc), C.byref(nm),
                              C.byref(ps), C.byref(pe), C.byref(pu), C.byref(pv)))
    n = nc.value

    def take(p, ctype, dtype):
        if n == 0:
            return np.zeros(0, dtype)
        # the array views the library's buffer, which is freed when the
        # array (and every view of it) is gone
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), shape=(n,))
        assert arr.dtype == dtype
        weakref.finalize(arr, L.rp_free, p.value)
        return arr

    return {"n_nodes": nn.value, "n_index": ni.value, "n_malformed": nm.value,
            "start": take(ps, C.c_int64, np.int64), "end": take(pe, C.c_int64, np.int64),
            "u": take(pu, C.c_int32, np.int32), "v": take(pv, C.c_int32, np.int32)}


class Graph:
    """A contact network held on one GPU (interval index + contacts)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @classmethod
    def load(cls, path, device=0):
        h = C.c_void_p()
        check(lib().rp_graph_load_text(str(path).encode(), device, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, start, end, u, v, n_nodes, device=0):
        start = np.ascontiguousarray(start, np.int64)
        end = np.ascontiguousarray(end, np.int64)
        u = np.ascontiguousarray(u, np.int32)
        v = np.ascontiguousarray(v, np.int32)
        h = C.c_void_p()
        check(lib().rp_graph_from_arrays(_ptr(start), _ptr(end), _ptr(u), _ptr(v), len(start), int(n_nodes),
                                         device, C.byref(h)))
        return cls(h.value)

    @property
    def info(self):
        gi = _lib.GraphInfo()
        check(lib().rp_graph_get_info(self._h, C.byref(gi)))
        return {k: getattr(gi, k) for k, _ in gi._fields_}

    @property
    def n_nodes(self):
        return self.info["n_nodes"]

    def close(self):
        if self._h and self._h.value:
            lib().rp_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_networks(networks):
    """Concatenates independent networks (dicts with start, end, u, v,
    n_nodes) into one union contact list; returns (start, end, u, v,
    n_nodes, offsets) with network k's nodes at [offsets[k], offsets[k+1])."""
    offsets = np.zeros(len(networks) + 1, np.int64)
    for k, net in enumerate(networks):
        offsets[k + 1] = offsets[k] + int(net["n_nodes"])
    if offsets[-1] >= 2 ** 31:
        raise ValueError("the batch exceeds 2^31 nodes")
    start = np.concatenate([np.asarray(n["start"], np.int64) for n in networks])
    end = np.concatenate([np.asarray(n["end"], np.int64) for n in networks])
    u = np.concatenate([np.asarray(n["u"], np.int64) + offsets[k] for k, n in enumerate(networks)]).astype(np.int32)
    v = np.concatenate([np.asarray(n["v"], np.int64) + offsets[k] for k, n in enumerate(networks)]).astype(np.int32)
    return start, end, u, v, int(offsets[-1]), offsets.astype(np.int32)


def window_csr(graph, ws, we, scale=1.0, weight="f32", ncls_cap=True):
    """Canonical symmetric CSR of window [ws, we) built on the GPU.

    weight "f32": (float)overlap*scale merged in hit order (the reference's
    build_csr_from_intervals); "i32": integer contact-seconds.
    Returns (row_ptr, col, val, n_hits)."""
    n = graph.n_nodes
    kind = 0 if weight == "f32" else 1
    row_ptr = np.zeros(n + 1, np.int32)
    nnz, nh = C.c_int64(), C.c_int64()
    cap = 1
    while True:
        col = np.zeros(cap, np.int32)
        val = np.zeros(cap, np.float32 if kind == 0 else np.int32)
        st = lib().rp_window_csr(graph._h, int(ws), int(we), float(scale), kind, 1 if ncls_cap else 0,
                                 _ptr(row_ptr), _ptr(col), _ptr(val), cap, C.byref(nnz), C.byref(nh))
        if st == 6 and nnz.value > cap:  # RP_ERR_RANGE: grow to the reported size
            cap = nnz.value
            continue
        check(st)
        return row_ptr, col[: nnz.value], val[: nnz.value], nh.value


class Simulation:
    """One replay configuration on a Graph (device state owned here).

    Keyword arguments mirror rp_params / the CLI flags:
      M (n_replicas), iterations (n_steps), step_size, start_time, window
      (static network duration), transition ("countdown" | "geometric"),
      path ("auto" | "plain" | "batched"), csr ("per-step" | "prebuilt"),
      seed, exposed_duration, infectious_duration, resistant_duration,
      infect_prob, initial_infected, initial_count, beta, beta_per_replica,
      susceptibility, p_ei, p_ir, p_rs, has_exposed, ir_to_s, ncls_cap,
      record_node_states.
    networks: optional node offsets (n_networks + 1) of independent networks
      batched in the graph (see batch_networks); counts then carry a network
      axis, (T+1, n_networks, M, 4).  A batch runs on the batched path with
      the hit cap off (ncls_cap defaults to False).
    """

    _ALIASES = {"M": "n_replicas", "iterations": "n_steps", "static_network_duration": "window",
                "time_step": "window"}

    def __init__(self, graph, networks=None, **kw):
        self.graph = graph
        p = _lib.Params()
        lib().rp_params_default(C.byref(p))
        self._keep = []
        if networks is not None:
            kw.setdefault("ncls_cap", False)
        for k, val in kw.items():
            k = self._ALIASES.get(k, k)
            if k == "transition":
                val = _lib.TRANSITION[val] if isinstance(val, str) else int(val)
            elif k == "path":
                val = _lib.PATH[val] if isinstance(val, str) else int(val)
            elif k == "csr":
                k, val = "csr_mode", (_lib.CSR_MODE[val] if isinstance(val, str) else int(val))
            elif k in ("beta_per_replica", "susceptibility"):
                if val is None:
                    continue
                arr = np.ascontiguousarray(val, np.float32)
                self._keep.append(arr)
                val = arr.ctypes.data
            elif k in ("ncls_cap", "has_exposed", "ir_to_s", "record_node_states"):
                val = int(bool(val))
            if not hasattr(p, k) or k == "struct_size":
                raise TypeError(f"unknown simulation parameter {k!r}")
            setattr(p, k, val)
        self.params = p
        h = C.c_void_p()
        if networks is None:
            self.n_networks = None
            check(lib().rp_sim_create(graph._h, C.byref(p), C.byref(h)))
        else:
            nf = np.ascontiguousarray(networks, np.int32)
            self._keep.append(nf)
            self.n_networks = len(nf) - 1
            check(lib().rp_sim_create_batch(graph._h, C.byref(p), _ptr(nf), self.n_networks, C.byref(h)))
        self._h = h
        self.M, self.T = p.n_replicas, p.n_steps

    def _shape(self, flat):
        if self.n_networks is None:
            return flat.reshape(self.T + 1, self.M, 4)
        return flat.reshape(self.T + 1, self.n_networks, self.M, 4)

    def _zeros(self):
        return np.zeros((self.T + 1) * (self.n_networks or 1) * self.M * 4, np.int32)

    @property
    def info(self):
        si = _lib.SimInfo()
        check(lib().rp_sim_get_info(self._h, C.byref(si)))
        return {k: getattr(si, k) for k, _ in si._fields_}

    def run(self, node_states=None):
        """Runs the replay; returns counts (T+1, M, 4) as (E, I, R, S)
        ((T+1, n_networks, M, 4) for a network batch).

        node_states: optional callable(step_index, timestamp, states[M, N])
        (requires record_node_states=True)."""
        counts = self._zeros()
        if node_states is not None:
            def _cb(user, step_index, ts, states, n, m):
                arr = np.ctypeslib.as_array(states, shape=(m * n,)).reshape(m, n).copy()
                return int(bool(node_states(step_index, ts, arr)))
            cb = _lib.STATE_CB(_cb)
        else:
            cb = _lib.STATE_CB()
        check(lib().rp_sim_run(self._h, _ptr(counts), cb, None))
        return self._shape(counts)

    def autotune(self, probe_steps=48):
        """Chooses the batched path's task height and staging depth per
        network-size bucket by timing the first probe_steps steps; returns
        the tuner's report (0 = default kept)."""
        r = _lib.TuneResult()
        check(lib().rp_sim_autotune(self._h, int(probe_steps), C.byref(r)))
        nb = r.n_buckets
        return {"buckets_log2": list(r.bucket_log2[:nb]), "rows_per_task": list(r.rows_per_task[:nb]),
                "stage_pairs": list(r.stage_pairs[:nb]), "probe_steps": r.probe_steps, "probes": r.probes,
                "ms_default": r.ms_default, "ms_tuned": r.ms_tuned}

    def run_text(self, write):
        """Runs the replay with node-state CSV lines formatted on the GPU;
        write(step_index, timestamp, data: bytes) receives them in chunks of
        whole lines (requires record_node_states=True).  Returns counts."""
        counts = self._zeros()

        def _cb(user, step_index, ts, text, n):
            return int(bool(write(step_index, ts, C.string_at(text, n))))
        cb = _lib.TEXT_CB(_cb)
        check(lib().rp_sim_run_text(self._h, _ptr(counts), cb, None))
        return self._shape(counts)

    def profile(self):
        """Device time per kernel group of one eager replay (CUDA events)."""
        pr = _lib.Profile()
        check(lib().rp_sim_profile(self._h, C.byref(pr)))
        return {k: getattr(pr, k) for k, _ in pr._fields_}

    def profile_steps(self):
        """Per-step device time (ms) of the exposure + transition kernels."""
        ms = np.zeros(max(self.T, 1), np.float32)
        check(lib().rp_sim_profile_steps(self._h, _ptr(ms)))
        return ms[: self.T]

    def enqueue(self, stream=None):
        """Enqueues the whole replay on a CUDA stream handle (int) without sync."""
        check(lib().rp_sim_enqueue(self._h, C.c_void_p(stream) if stream else None))

    def counts(self):
        counts = self._zeros()
        check(lib().rp_sim_counts(self._h, _ptr(counts)))
        return self._shape(counts)

    def timestamps(self):
        ts = np.zeros(self.T + 1, np.int64)
        check(lib().rp_sim_timestamps(self._h, _ptr(ts)))
        return ts

    def close(self):
        if self._h and self._h.value:
            lib().rp_sim_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
