"""The dense stress network: N = 5,000 nodes, 50M contacts whose endpoints
follow power-law node activity, 15 min steps over 30 days (2,880 steps),
16,384 replicas, SIR.  Hub rows hold thousands of CSR entries per window,
more than the infection kernel stages in shared memory at a time, so their
pairs are read from global memory.

A reduced instance with the same node count and the same contacts per window
(one day instead of 30: 96 steps, 64 replicas) is bit-identical to the
oracle.  The full instance is checked through properties that hold at any
size: every replica's compartments sum to N at every step, SIR counts are
monotone, the initial count is exact, and a shard of replicas run on its own
(with its replica offset) reproduces its slice of the full run.
"""
import numpy as np
import pytest

from replay_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200
    replay_b200.lib()
    return replay_b200


def _graph(rb, net):
    return rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])


@pytest.mark.parametrize("csr", ["per-step", "prebuilt"])
def test_reduced_dense_stress_matches_oracle(rb, oracle, csr):
    # one day at the full network's contact rate: about 40,000 hits per
    # window, hub rows above 3,000 entries
    net = synthetic.dense_stress(seed=6, n_contacts=1_666_667, days=1, steps=96, replicas=64)
    kw = dict(net["params"], M=64, iterations=96, beta=3e-5, initial_count=20, seed=11)
    g = _graph(rb, net)
    ws = int(kw["start_time"]) + 40 * 900
    rp, col, val, nh = rb.window_csr(g, ws, ws + 900, 1.0, "i32", False)
    assert np.diff(rp).max() > 1024  # a row larger than one staged chunk
    got = rb.Simulation(g, path="batched", csr=csr, **kw).run()
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], n_replicas=64,
                      n_steps=96, step_size=kw["step_size"], window=kw["window"],
                      start_time=kw["start_time"], transition=1, beta=kw["beta"], p_ir=kw["p_ir"],
                      has_exposed=0, initial_count=20, seed=11)
    np.testing.assert_array_equal(got, want)
    assert got[-1, :, 2].sum() > 0  # recoveries happened


@pytest.mark.parametrize("csr", ["per-step", "prebuilt"])
def test_dense_neighbourhoods_match_oracle(rb, oracle, csr):
    """Five percent initially infected on the dense network: in the first
    steps most susceptible replicas of a row are exposed with an infection
    bound near 1, so whole words reach the exact test (the one-pass word
    test as well as the per-replica one)."""
    net = synthetic.dense_stress(seed=6, n_contacts=1_666_667, days=1, steps=96, replicas=64)
    kw = dict(net["params"], M=64, iterations=24, initial_count=250, seed=13)
    g = _graph(rb, net)
    got = rb.Simulation(g, path="batched", csr=csr, **kw).run()
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], n_replicas=64,
                      n_steps=24, step_size=kw["step_size"], window=kw["window"],
                      start_time=kw["start_time"], transition=1, beta=kw["beta"], p_ir=kw["p_ir"],
                      has_exposed=0, initial_count=250, seed=13)
    np.testing.assert_array_equal(got, want)
    # the epidemic takes off in every replica from the first steps
    assert (got[0, :, 3] - got[2, :, 3]).min() > 0
    assert (got[0, :, 3] - got[2, :, 3]).mean() > 20


def test_full_dense_stress_properties_and_shard(rb):
    net = synthetic.dense_stress()
    p = dict(net["params"])
    n, m, T = net["n_nodes"], p["M"], p["iterations"]
    assert (n, m, T) == (5000, 16384, 2880)
    g = _graph(rb, net)
    full = rb.Simulation(g, path="batched", **p).run()
    assert full.shape == (T + 1, m, 4)
    # columns: exposed, infectious, resistant, susceptible
    assert (full.sum(axis=2) == n).all()
    assert (full[:, :, 0] == 0).all()  # SIR: no exposed state
    assert (full[0, :, 1] == 5).all()
    assert (np.diff(full[:, :, 2].astype(np.int64), axis=0) >= 0).all()  # R never decreases
    assert (np.diff(full[:, :, 3].astype(np.int64), axis=0) <= 0).all()  # S never increases
    assert full[-1, :, 2].mean() > 5  # the epidemic spreads in some replicas
    off, cnt = 4096, 512
    shard = rb.Simulation(g, path="batched", csr="prebuilt", **dict(p, M=cnt),
                          replica_offset=off).run()
    np.testing.assert_array_equal(shard, full[:, off:off + cnt])
