"""GPU parity: the CUDA path against the C oracle on the same seeded inputs.

Window CSRs, exposures, and whole replays (counts of every step) must be
bit-identical: integer/byte work is exact, and every float operation on the
device uses the same correctly rounded sequence as the oracle.
"""
import numpy as np
import pytest

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


def _index(oracle, net):
    return oracle.sorted_index(net["start"], net["end"], net["u"], net["v"])


@pytest.mark.parametrize("seed,negative", [(0, False), (1, False), (2, True), (3, True)])
def test_window_csr_f32_matches_oracle(rb, oracle, seed, negative):
    from replay_b200 import synthetic
    net = synthetic.tiny(seed=seed, negative=negative)
    g = _graph(rb, net)
    ss, se, su, sv, perm, nl = _index(oracle, net)
    assert g.info["nlists"] == nl
    t0 = net["t0"]
    for k, W in enumerate([600, 1800, 3600, 7200]):
        for ws in range(t0 - W, t0 + 6 * 3600 + W, W):
            for scale in (1.0, np.float32(1 / 3)):
                for cap in (True, False):
                    rp, col, val, nh = rb.window_csr(g, ws, ws + W, scale, "f32", cap)
                    hits = oracle.window_hits(ss, se, nl if cap else len(ss), ws, ws + W)
                    orp, ocol, oval = oracle.csr_f32(ss, se, su, sv, hits, net["n_nodes"], ws, ws + W,
                                                     np.float32(scale))
                    assert nh == len(hits)
                    np.testing.assert_array_equal(rp, orp)
                    np.testing.assert_array_equal(col, ocol)
                    np.testing.assert_array_equal(val.view(np.int32), oval.view(np.int32))


def test_window_csr_hit_cap_binds(rb, oracle):
    # five mutually overlapping, non-nested contacts: nlists = 4, the
    # reference query returns only 4 hits.
    s = np.array([0, 10, 20, 30, 40], np.int64) + 946684800
    e = s + 100
    u = np.array([0, 1, 2, 3, 4], np.int32)
    v = np.array([5, 6, 7, 8, 9], np.int32)
    g = rb.Graph.from_arrays(s, e, u, v, 10)
    assert g.info["nlists"] == 4
    rp, col, val, nh = rb.window_csr(g, 946684800, 946684800 + 3600, 1.0, "f32", True)
    assert nh == 4 and len(col) == 8
    rp, col, val, nh = rb.window_csr(g, 946684800, 946684800 + 3600, 1.0, "f32", False)
    assert nh == 5 and len(col) == 10


@pytest.mark.parametrize("seed", [4, 5])
def test_window_csr_i32_matches_oracle(rb, oracle, seed):
    from replay_b200 import synthetic
    net = synthetic.tiny(seed=seed, n_nodes=60, n_contacts=3000, max_dur=20000)
    g = _graph(rb, net)
    ss, se, su, sv, perm, nl = _index(oracle, net)
    for ws in range(net["t0"] - 3600, net["t0"] + 7 * 3600, 1800):
        rp, col, val, nh = rb.window_csr(g, ws, ws + 3600, 1.0, "i32", False)
        hits = oracle.window_hits(ss, se, len(ss), ws, ws + 3600)
        orp, ocol, oval = oracle.csr_i32(ss, se, su, sv, hits, net["n_nodes"], ws, ws + 3600)
        np.testing.assert_array_equal(rp, orp)
        np.testing.assert_array_equal(col, ocol)
        np.testing.assert_array_equal(val, oval)


def _oracle_kw(sim_kw):
    kw = dict(sim_kw)
    m = {"M": "n_replicas", "iterations": "n_steps"}
    out = {}
    for k, v in kw.items():
        k = m.get(k, k)
        if k == "transition":
            v = 0 if v == "countdown" else 1
        if k in ("path", "csr"):
            continue
        if isinstance(v, bool):
            v = int(v)
        out[k] = v
    return out


COUNTDOWN_CASES = [
    dict(M=37, iterations=30, step_size=1800.0, window=1800, initial_infected=0.1, infect_prob=0.3,
         exposed_duration=3600, infectious_duration=7200, resistant_duration=3600),
    dict(M=20, iterations=25, step_size=1200.0, window=3600, initial_infected=0.2, infect_prob=0.5,
         exposed_duration=0, infectious_duration=5000, resistant_duration=0),
    dict(M=16, iterations=20, step_size=3600.0, window=3600, initial_count=3, infect_prob=1.0,
         exposed_duration=3600, infectious_duration=3600, resistant_duration=100000000),
    # long durations: more than 256 countdown values (16-bit codes on the batched path)
    dict(M=40, iterations=140, step_size=1800.0, window=1800, initial_infected=0.05, infect_prob=0.2,
         exposed_duration=100000, infectious_duration=200000, resistant_duration=100000000),
]


@pytest.mark.parametrize("case", range(len(COUNTDOWN_CASES)))
@pytest.mark.parametrize("path,csr", [("plain", "per-step"), ("plain", "prebuilt"), ("batched", "per-step"),
                                      ("batched", "prebuilt")])
def test_countdown_replay_matches_oracle(rb, oracle, case, path, csr):
    from replay_b200 import synthetic
    net = synthetic.tiny(seed=10 + case, n_nodes=50, n_contacts=800)
    kw = dict(COUNTDOWN_CASES[case], start_time=net["t0"], seed=99 + case, transition="countdown")
    g = _graph(rb, net)
    got = rb.Simulation(g, path=path, csr=csr, **kw).run()
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], **_oracle_kw(kw))
    np.testing.assert_array_equal(got, want)


GEOMETRIC_CASES = [
    dict(M=70, iterations=30, beta=4e-4, p_ei=0.2, p_ir=0.1, initial_count=3),
    dict(M=33, iterations=30, beta=8e-4, p_ir=0.15, has_exposed=False, initial_infected=0.05),
    dict(M=64, iterations=40, beta=6e-4, p_ei=0.3, p_ir=0.2, p_rs=0.1, initial_count=4),
    dict(M=40, iterations=30, beta=5e-4, p_ir=0.2, has_exposed=False, ir_to_s=True, initial_count=5),
    dict(M=96, iterations=24, beta=3e-4, p_ei=0.25, p_ir=0.1, initial_count=2, window=7200),
    dict(M=45, iterations=20, beta=1e-3, p_ei=1.0, p_ir=3e-9, p_rs=0.5, initial_count=6),
]


@pytest.mark.parametrize("case", range(len(GEOMETRIC_CASES)))
@pytest.mark.parametrize("path,csr", [("plain", "per-step"), ("batched", "per-step"), ("batched", "prebuilt")])
def test_geometric_replay_matches_oracle(rb, oracle, case, path, csr):
    from replay_b200 import synthetic
    net = synthetic.tiny(seed=20 + case, n_nodes=80, n_contacts=1500)
    kw = dict(step_size=1800.0, window=1800, start_time=net["t0"], seed=7 + case, transition="geometric")
    kw.update(GEOMETRIC_CASES[case])
    rng = np.random.default_rng(case)
    if case == 2:
        kw["beta_per_replica"] = (rng.random(kw["M"]) * 1e-3).astype(np.float32)
        kw["susceptibility"] = rng.uniform(0.5, 1.5, net["n_nodes"]).astype(np.float32)
    g = _graph(rb, net)
    got = rb.Simulation(g, path=path, csr=csr, **kw).run()
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], **_oracle_kw(kw))
    np.testing.assert_array_equal(got, want)
    assert got[-1, :, :].sum() == kw["M"] * net["n_nodes"]


def test_batched_equals_plain_small_seir(rb):
    from replay_b200 import synthetic
    net = synthetic.small_seir(seed=1)
    p = dict(net["params"], M=256, iterations=48)
    g = _graph(rb, net)
    a = rb.Simulation(g, path="plain", **p).run()
    b = rb.Simulation(g, path="batched", **p).run()
    c = rb.Simulation(g, path="batched", csr="prebuilt", **p).run()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)


def test_node_states_callback(rb, oracle):
    from replay_b200 import synthetic
    net = synthetic.tiny(seed=31, n_nodes=30, n_contacts=300)
    kw = dict(M=9, iterations=6, step_size=1800.0, window=1800, start_time=net["t0"], seed=3,
              transition="geometric", beta=1e-3, p_ei=0.3, p_ir=0.2, initial_count=2)
    g = _graph(rb, net)
    seen = []
    sim = rb.Simulation(g, record_node_states=True, **kw)
    counts = sim.run(node_states=lambda k, ts, st: seen.append(st) and 0)
    want_c, want_s = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"],
                                node_states=True, **_oracle_kw(kw))
    np.testing.assert_array_equal(counts, want_c)
    np.testing.assert_array_equal(np.stack(seen), want_s)


@pytest.mark.parametrize("negative", [False, True])
def test_device_index_matches_oracle_across_sort_tiles(rb, oracle, negative):
    """300k contacts (73 radix tiles, 74 nesting chunks) with many exact
    ties and nested intervals: nlists and window CSRs match the oracle."""
    rng = np.random.default_rng(7 + negative)
    n, nodes = 300_000, 5000
    base = -3 * 86400 if negative else 946684800
    start = base + rng.integers(0, 86400, n) // 60 * 60  # minute grid: many equal starts
    end = start + rng.choice([1, 60, 600, 3600, 7200, 40000], n)  # few durations: ties and nesting
    u = rng.integers(0, nodes, n).astype(np.int32)
    v = ((u + 1 + rng.integers(0, nodes - 1, n)) % nodes).astype(np.int32)
    g = rb.Graph.from_arrays(start, end, u, v, nodes)
    ss, se, su, sv, perm, nl = oracle.sorted_index(start, end, np.minimum(u, v), np.maximum(u, v))
    assert g.info["nlists"] == nl
    for ws in (base, base + 3 * 3600 + 17, base + 20 * 3600):
        for cap in (True, False):
            rp, col, val, nh = rb.window_csr(g, ws, ws + 3600, 1.0, "f32", cap)
            hits = oracle.window_hits(ss, se, nl if cap else len(ss), ws, ws + 3600)
            orp, ocol, oval = oracle.csr_f32(ss, se, su, sv, hits, nodes, ws, ws + 3600, np.float32(1.0))
            assert nh == len(hits)
            np.testing.assert_array_equal(rp, orp)
            np.testing.assert_array_equal(col, ocol)
            np.testing.assert_array_equal(val.view(np.int32), oval.view(np.int32))
