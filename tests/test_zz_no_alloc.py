"""rp_window_csr_noalloc against rp_window_csr, through the C ABI.

Collected last (tests/conftest.py keeps this file at the end).  Calls in a
row on different windows, including windows that start before 1970 (the
mirrored query of the interval index), must each reproduce the allocating
entry point's CSR exactly, and the calls must not change the device's free
memory.  Device-wide free memory can also move because of other work on a
shared GPU, so that check is retried a few times before it fails.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(L, g, ws, we, scale, kind, cap, d_rp, d_ent, capacity, stream):
    nnz, nh = C.c_int64(), C.c_int64()
    st = L.rp_window_csr_noalloc(g._h, ws, we, scale, kind, cap, d_rp.data_ptr(), d_ent.data_ptr(), capacity,
                                 C.byref(nnz), C.byref(nh), stream)
    return st, nnz.value, nh.value


def _check_windows(L, rb, g, n, windows, capacity):
    import torch
    d_rp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    d_ent = torch.empty(2 * capacity, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    total = 0
    for ws, we, scale, kind, cap in windows:
        # two calls in a row on the same window: the scratch keeps the last
        # call's contents, and the second call must not depend on them
        for _ in range(2):
            d_rp.fill_(-7)
            st, nnz, nh = _noalloc(L, g, ws, we, scale, kind, cap, d_rp, d_ent, capacity, stream)
            assert st == 0, L.rp_last_error()
            torch.cuda.synchronize()
            rp, col, val, want_nh = rb.window_csr(g, ws, we, scale, "f32" if kind == 0 else "i32", bool(cap))
            got_rp = d_rp.cpu().numpy()
            pairs = d_ent[:2 * nnz].cpu().numpy().reshape(-1, 2)
            np.testing.assert_array_equal(got_rp, rp)
            assert nnz == len(col) and nh == want_nh
            np.testing.assert_array_equal(pairs[:, 0], col)
            np.testing.assert_array_equal(pairs[:, 1], val.view(np.int32))
            total += nnz
    return total


def _free_memory_unchanged(call, tries=5):
    import torch
    for _ in range(tries):
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()[0]
        call()
        torch.cuda.synchronize()
        if torch.cuda.mem_get_info()[0] == before:
            return True
    return False


def test_noalloc_window_csr_matches_allocating_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    from replay_b200 import synthetic
    L = rb.lib()
    net = synthetic.tiny(seed=41, n_nodes=300, n_contacts=6000, span=8 * 3600, max_dur=7000)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    t0 = net["t0"]
    windows = [(t0 + 1800, t0 + 5400, 1.0, 0, 1),
               (t0 + 7200, t0 + 9000, float(np.float32(1 / 3)), 0, 0),
               (t0 - 600, t0 + 3000, 1.0, 1, 1)]
    assert _check_windows(L, rb, g, net["n_nodes"], windows, 2 * len(net["start"])) > 0

    # contacts on both sides of 1970: windows with ws < 0 take the mirrored query
    neg = synthetic.tiny(seed=44, n_nodes=200, n_contacts=5000, span=8 * 3600, max_dur=7000, negative=True)
    gn = rb.Graph.from_arrays(neg["start"], neg["end"], neg["u"], neg["v"], neg["n_nodes"])
    windows = [(-7200, -3600, 1.0, 1, 1), (-1800, 1800, 1.0, 0, 1), (-5400, -1800, float(np.float32(0.5)), 0, 0),
               (600, 4200, 1.0, 1, 0)]
    assert _check_windows(L, rb, gn, neg["n_nodes"], windows, 2 * len(neg["start"])) > 0

    # no device allocation or free on a call (the scratch is static)
    d_rp = torch.empty(net["n_nodes"] + 1, dtype=torch.int32, device="cuda")
    d_ent = torch.empty(4 * len(net["start"]), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        st, _, _ = _noalloc(L, g, t0 + 1800, t0 + 5400, 1.0, 0, 1, d_rp, d_ent, 2 * len(net["start"]), stream)
        assert st == 0, L.rp_last_error()
    assert _free_memory_unchanged(call)


def test_noalloc_rejects_oversized_requests():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    from replay_b200 import synthetic
    L = rb.lib()
    net = synthetic.tiny(seed=42, n_nodes=70000, n_contacts=1000)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    d_rp = torch.empty(net["n_nodes"] + 1, dtype=torch.int32, device="cuda")
    d_ent = torch.empty(4000, dtype=torch.int32, device="cuda")
    st, _, _ = _noalloc(L, g, net["t0"], net["t0"] + 3600, 1.0, 0, 1, d_rp, d_ent, 2000,
                        torch.cuda.current_stream().cuda_stream)
    assert st == 6 and b"at most 65536" in L.rp_last_error()
    # capacity too small for the CSR: RP_ERR_RANGE with nnz reported
    net = synthetic.tiny(seed=43, n_nodes=50, n_contacts=2000)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    d_rp = torch.empty(51, dtype=torch.int32, device="cuda")
    nnz, nh = C.c_int64(), C.c_int64()
    st = L.rp_window_csr_noalloc(g._h, net["t0"], net["t0"] + 3600, 1.0, 0, 1, d_rp.data_ptr(),
                                 d_ent.data_ptr(), 1, C.byref(nnz), C.byref(nh),
                                 torch.cuda.current_stream().cuda_stream)
    assert st == 6 and nnz.value > 1
    # the caller's current device is left as it was
    assert torch.cuda.current_device() == 0
