"""Independent networks of uneven size batched into one replay.

The batch is the union graph with per-network node ranges; every count of
every (step, network, replica) must equal the oracle's run of the same
union with the same partition (exact-k seeding draws per network on its
own stream; all other draws are keyed by the union's node index)."""
import numpy as np
import pytest

from replay_b200 import synthetic


def _nets(seed=60, sizes=(30, 85, 50, 120)):
    nets = []
    for k, n in enumerate(sizes):
        net = synthetic.tiny(seed=seed + k, n_nodes=n, n_contacts=12 * n, span=12 * 3600)
        nets.append(net)
    return nets


def _union(nets):
    import replay_b200 as rb
    return rb.batch_networks(nets)


def test_batch_networks_offsets_and_oracle_conservation(oracle):
    nets = _nets()
    s, e, u, v, n, off = _union(nets)
    assert list(off) == [0, 30, 115, 165, 285] and n == 285
    for k, net in enumerate(nets):
        sel = slice(int(sum(len(x["u"]) for x in nets[:k])), int(sum(len(x["u"]) for x in nets[:k + 1])))
        assert u[sel].min() >= off[k] and v[sel].max() < off[k + 1]
    kw = dict(n_replicas=40, n_steps=20, step_size=1800.0, window=1800, start_time=nets[0]["t0"], transition=1,
              seed=3, beta=8e-4, p_ei=0.3, p_ir=0.2, initial_count=4, ncls_cap=0)
    c = oracle.run(s, e, u, v, n, net_first=off, **kw)
    assert c.shape == (21, 4, 40, 4)
    np.testing.assert_array_equal(c.sum(axis=3), np.broadcast_to(np.diff(off)[None, :, None], (21, 4, 40)))
    np.testing.assert_array_equal(c[0, :, :, 1], 4)  # exactly 4 infectious per (network, replica) at t0
    # a one-network partition reproduces the unpartitioned run
    one = oracle.run(s, e, u, v, n, net_first=np.array([0, n], np.int32), **kw)
    np.testing.assert_array_equal(one[:, 0], oracle.run(s, e, u, v, n, **kw))


BATCH_CASES = [
    dict(M=70, iterations=24, beta=8e-4, p_ei=0.3, p_ir=0.2, initial_count=3),
    dict(M=40, iterations=20, beta=1e-3, p_ir=0.15, has_exposed=False, initial_infected=0.05, p_rs=0.1),
    dict(M=130, iterations=16, beta=6e-4, p_ei=0.25, p_ir=0.1, initial_count=5, ir_to_s=True),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(BATCH_CASES)))
@pytest.mark.parametrize("csr", ["per-step", "prebuilt"])
def test_batch_matches_oracle(oracle, case, csr):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    nets = _nets(seed=70 + case)
    s, e, u, v, n, off = _union(nets)
    kw = dict(step_size=1800.0, window=1800, start_time=nets[0]["t0"], seed=11 + case, transition="geometric")
    kw.update(BATCH_CASES[case])
    g = rb.Graph.from_arrays(s, e, u, v, n)
    got = rb.Simulation(g, networks=off, path="batched", csr=csr, **kw).run()
    okw = {"M": "n_replicas", "iterations": "n_steps"}
    want = oracle.run(s, e, u, v, n, net_first=off, ncls_cap=0,
                      **{okw.get(k, k): (1 if k == "transition" else (int(val) if isinstance(val, bool) else val))
                         for k, val in kw.items()})
    assert got.shape == want.shape == (kw["iterations"] + 1, len(nets), kw["M"], 4)
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_batch_argument_errors():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    nets = _nets()
    s, e, u, v, n, off = _union(nets)
    g = rb.Graph.from_arrays(s, e, u, v, n)
    kw = dict(M=32, iterations=4, transition="geometric", beta=1e-4, p_ir=0.1, start_time=nets[0]["t0"])
    with pytest.raises(rb.ReplayError, match="hit cap"):
        rb.Simulation(g, networks=off, ncls_cap=True, **kw)
    with pytest.raises(rb.ReplayError, match="offsets"):
        rb.Simulation(g, networks=off[:-1], **kw)
    with pytest.raises(rb.ReplayError, match="smallest network"):
        rb.Simulation(g, networks=off, initial_count=31, **kw)
    with pytest.raises(rb.ReplayError, match="batched"):
        rb.Simulation(g, networks=off, **dict(kw, path="plain"))


@pytest.mark.gpu
@pytest.mark.parametrize("csr", ["per-step", "prebuilt"])
def test_countdown_batch_matches_oracle(oracle, csr):
    """The reference's countdown rules on a batch of uneven networks."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    nets = _nets(seed=80)
    s, e, u, v, n, off = _union(nets)
    kw = dict(M=70, iterations=24, step_size=1800.0, window=1800, start_time=nets[0]["t0"], seed=13,
              transition="countdown", initial_count=3, infect_prob=0.3, exposed_duration=3600,
              infectious_duration=7200, resistant_duration=5400)
    g = rb.Graph.from_arrays(s, e, u, v, n)
    got = rb.Simulation(g, networks=off, path="batched", csr=csr, **kw).run()
    okw = {"M": "n_replicas", "iterations": "n_steps"}
    want = oracle.run(s, e, u, v, n, net_first=off, ncls_cap=0,
                      **{okw.get(k, k): (0 if k == "transition" else val) for k, val in kw.items()})
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_autotune_keeps_results_and_reports():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    nets = _nets(seed=90, sizes=(40, 300, 70, 1100, 520))
    s, e, u, v, n, off = _union(nets)
    g = rb.Graph.from_arrays(s, e, u, v, n)
    kw = dict(M=96, iterations=30, step_size=1800.0, window=1800, start_time=nets[0]["t0"], seed=5,
              transition="geometric", beta=7e-4, p_ei=0.3, p_ir=0.15, initial_count=3)
    sim = rb.Simulation(g, networks=off, **kw)
    before = sim.run()
    rep = sim.autotune(probe_steps=10)
    assert sorted(rep["buckets_log2"], reverse=True) == rep["buckets_log2"] == [10, 9, 8, 6, 5]
    assert rep["probes"] == 1 + (8 + 2) * 5 and rep["ms_tuned"] <= rep["ms_default"]
    assert all(r in (0, 32, 64, 128, 256, 512, 1024, 2048, 4096) for r in rep["rows_per_task"])
    assert all(r in (0, 192, 384) for r in rep["stage_pairs"])
    np.testing.assert_array_equal(sim.run(), before)
