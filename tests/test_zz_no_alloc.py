"""rp_window_csr_noalloc against rp_window_csr, through the C ABI.

Collected last (file name).  Calls in a row on different windows must each
reproduce the allocating entry point's CSR exactly, and every call after
the first (which may load the module holding the scratch) must leave the
device's free memory unchanged.
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


def test_noalloc_window_csr_matches_allocating_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    from replay_b200 import synthetic
    L = rb.lib()
    net = synthetic.tiny(seed=41, n_nodes=300, n_contacts=6000, span=8 * 3600, max_dur=7000)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    n = net["n_nodes"]
    capacity = 2 * len(net["start"])
    d_rp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    d_ent = torch.empty(2 * capacity, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()

    windows = [(net["t0"] + 1800, net["t0"] + 5400, 1.0, 0, 1),
               (net["t0"] + 7200, net["t0"] + 9000, float(np.float32(1 / 3)), 0, 0),
               (net["t0"] - 600, net["t0"] + 3000, 1.0, 1, 1)]
    for i, (ws, we, scale, kind, cap) in enumerate(windows):
        free_before = torch.cuda.mem_get_info()[0]
        st, nnz, nh = _noalloc(L, g, ws, we, scale, kind, cap, d_rp, d_ent, capacity, stream)
        assert st == 0, L.rp_last_error()
        torch.cuda.synchronize()
        if i > 0:  # the first call may load the module that holds the scratch
            assert torch.cuda.mem_get_info()[0] == free_before
        rp, col, val, want_nh = rb.window_csr(g, ws, we, scale, "f32" if kind == 0 else "i32", bool(cap))
        got_rp = d_rp.cpu().numpy()
        pairs = d_ent[:2 * nnz].cpu().numpy().reshape(-1, 2)
        np.testing.assert_array_equal(got_rp, rp)
        assert nnz == len(col) and nh == want_nh
        np.testing.assert_array_equal(pairs[:, 0], col)
        np.testing.assert_array_equal(pairs[:, 1], val.view(np.int32))
    assert nnz > 0


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
