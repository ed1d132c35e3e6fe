"""ctypes binding of libreplay (include/replay.h).

The shared library is built in-tree (replay_b200/lib/libreplay.so) by
`make -C replay_b200/csrc`; importing fails loudly when it is missing --
there is no CPU fallback.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libreplay.so")
CLI_PATH = os.path.join(_HERE, "bin", "replay")

RP_OK = 0
STATUS_NAMES = {0: "RP_OK", 1: "RP_ERR_ARG", 2: "RP_ERR_IO", 3: "RP_ERR_PARSE", 4: "RP_ERR_NOMEM",
                5: "RP_ERR_CUDA", 6: "RP_ERR_RANGE", 7: "RP_ERR_DEVICE"}

TRANSITION = {"countdown": 0, "geometric": 1}
PATH = {"auto": 0, "plain": 1, "batched": 2}
CSR_MODE = {"per-step": 0, "prebuilt": 1}


class GraphInfo(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("n_index", C.c_int32), ("n_contacts", C.c_int64),
                ("nlists", C.c_int64), ("n_malformed", C.c_int64), ("t_min", C.c_int64),
                ("t_max", C.c_int64), ("n_classes", C.c_int32), ("device", C.c_int32),
                ("prep_ms", C.c_double), ("build_ms", C.c_double)]


class Params(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("n_replicas", C.c_int32),
        ("n_steps", C.c_int32),
        ("step_size", C.c_float),
        ("start_time", C.c_int64),
        ("window", C.c_int64),
        ("transition", C.c_int32),
        ("path", C.c_int32),
        ("csr_mode", C.c_int32),
        ("ncls_cap", C.c_int32),
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
        ("record_node_states", C.c_int32),
        ("replica_offset", C.c_int32),
    ]


class SimInfo(C.Structure):
    _fields_ = [("path", C.c_int32), ("words", C.c_int32), ("n_windows", C.c_int32),
                ("kernels_per_run", C.c_int32), ("max_candidates", C.c_int64),
                ("prebuilt_nnz", C.c_int64), ("device_bytes", C.c_int64), ("nnz_total", C.c_int64),
                ("setup_ms", C.c_double), ("alloc_ms", C.c_double), ("prebuild_ms", C.c_double),
                ("capture_ms", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("build_ms", C.c_double), ("spmv_ms", C.c_double),
                ("step_ms", C.c_double), ("other_ms", C.c_double), ("step_launches", C.c_int32),
                ("spmv_launches", C.c_int32), ("build_launches", C.c_int32), ("kernels", C.c_int32)]


STATE_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_uint8), C.c_int32,
                       C.c_int32)

# Every entry point of include/replay.h with its ctypes signature.
class TuneResult(C.Structure):
    _fields_ = [("n_buckets", C.c_int32), ("bucket_log2", C.c_int32 * 32), ("rows_per_task", C.c_int32 * 32),
                ("stage_pairs", C.c_int32 * 32), ("probe_steps", C.c_int32), ("probes", C.c_int32),
                ("ms_default", C.c_double), ("ms_tuned", C.c_double)]


TEXT_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_char), C.c_size_t)

SIGNATURES = {
    "rp_last_error": ([], C.c_char_p),
    "rp_version": ([], C.c_char_p),
    "rp_release_cached_memory": ([], None),
    "rp_graph_load_text": ([C.c_char_p, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "rp_graph_from_arrays": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int,
                              C.POINTER(C.c_void_p)], C.c_int),
    "rp_parse_contacts": ([C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                           C.POINTER(C.c_int64), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                           C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)], C.c_int),
    "rp_free": ([C.c_void_p], None),
    "rp_graph_get_info": ([C.c_void_p, C.POINTER(GraphInfo)], C.c_int),
    "rp_graph_free": ([C.c_void_p], None),
    "rp_window_csr": ([C.c_void_p, C.c_int64, C.c_int64, C.c_float, C.c_int32, C.c_int32, C.c_void_p,
                       C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    "rp_window_csr_noalloc": ([C.c_void_p, C.c_int64, C.c_int64, C.c_float, C.c_int32, C.c_int32, C.c_void_p,
                               C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_void_p],
                              C.c_int),
    "rp_params_default": ([C.POINTER(Params)], None),
    "rp_sim_create": ([C.c_void_p, C.POINTER(Params), C.POINTER(C.c_void_p)], C.c_int),
    "rp_sim_create_batch": ([C.c_void_p, C.POINTER(Params), C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)],
                            C.c_int),
    "rp_sim_free": ([C.c_void_p], None),
    "rp_sim_autotune": ([C.c_void_p, C.c_int32, C.POINTER(TuneResult)], C.c_int),
    "rp_sim_run": ([C.c_void_p, C.c_void_p, STATE_CB, C.c_void_p], C.c_int),
    "rp_sim_run_text": ([C.c_void_p, C.c_void_p, TEXT_CB, C.c_void_p], C.c_int),
    "rp_sim_enqueue": ([C.c_void_p, C.c_void_p], C.c_int),
    "rp_sim_counts": ([C.c_void_p, C.c_void_p], C.c_int),
    "rp_sim_timestamps": ([C.c_void_p, C.c_void_p], C.c_int),
    "rp_sim_get_info": ([C.c_void_p, C.POINTER(SimInfo)], C.c_int),
    "rp_sim_profile": ([C.c_void_p, C.POINTER(Profile)], C.c_int),
    "rp_sim_profile_steps": ([C.c_void_p, C.c_void_p], C.c_int),
    "rp_meanfield_create": ([C.c_void_p, C.POINTER(Params), C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
    "rp_meanfield_free": ([C.c_void_p], None),
    "rp_meanfield_forward": ([C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_float, C.c_float, C.c_float,
                              C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "rp_meanfield_backward": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
                               C.c_int),
    "rp_exposure_spmv_f32": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                              C.c_void_p], C.c_int),
    "rp_exposure_spmm_packed": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                 C.c_void_p], C.c_int),
}

_LIB = None


class ReplayError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def lib():
    """Loads libreplay.so (raises if the extension is not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libreplay is not built ({LIB_PATH} missing); run "
                              "`make -C replay_b200/csrc` or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = L
    return _LIB


def check(status):
    if status != RP_OK:
        msg = lib().rp_last_error()
        raise ReplayError(status, msg.decode() if msg else "")
