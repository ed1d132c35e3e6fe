"""Bit-exact oracle parity on the benchmark's own workloads.

Every count of every step of every replica must equal the C oracle's:
  * the replica sweep (N = 100,000 in 100 communities, 20M contacts, all
    336 one-hour steps) at full node and contact count, on 64 replicas
    taken from the top of the beta sweep (replica offset 4,032, the largest
    epidemics), with window CSRs built per step and prebuilt;
  * the small SEIR workload at full size (N = 1,000, 50,000 contacts, 168
    steps, 1,000 replicas) in geometric mode on the plain and batched paths,
    and in the reference's countdown mode (its own rules) on every path;
  * networks of the uneven batch sampled across its 500..50,000-node range,
    batched into one replay over all 1,440 half-hour steps.
The replays follow the reference's step loop (tool/gpu_cpu_temporal_sim.cu:
859-1096); the oracle restates it function by function.
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


def _oracle_kw(p, **extra):
    out = dict(n_replicas=p["M"], n_steps=p["iterations"], step_size=p["step_size"], window=p["window"],
               start_time=p["start_time"], transition=0 if p["transition"] == "countdown" else 1,
               seed=p.get("seed", 1))
    for k in ("beta", "beta_per_replica", "p_ei", "p_ir", "p_rs", "initial_count", "initial_infected",
              "infect_prob", "exposed_duration", "infectious_duration", "resistant_duration", "replica_offset",
              "ncls_cap", "has_exposed", "ir_to_s"):
        if k in p:
            v = p[k]
            out[k] = int(v) if isinstance(v, bool) else v
    out.update(extra)
    return out


@pytest.fixture(scope="module")
def sweep():
    return synthetic.replica_sweep()


@pytest.fixture(scope="module")
def sweep_top64(sweep, oracle):
    net = sweep
    off, M = 4096 - 64, 64
    p = dict(net["params"], M=M, replica_offset=off, ncls_cap=True,
             beta_per_replica=net["params"]["beta_per_replica"][off:off + M])
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], **_oracle_kw(p))
    return p, want


@pytest.mark.parametrize("csr", ["per-step", "prebuilt"])
def test_replica_sweep_full_network_matches_oracle(rb, sweep, sweep_top64, csr):
    p, want = sweep_top64
    net = sweep
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    got = rb.Simulation(g, path="batched", csr=csr, **p).run()
    assert got.shape == (337, 64, 4)
    np.testing.assert_array_equal(got, want)
    # the top of the sweep is a large epidemic: most replicas infect
    # thousands of nodes, so every kernel branch (bound test, exact test,
    # every flow) is exercised at this scale
    assert np.median(100_000 - want[-1, :, 3]) > 1000


@pytest.fixture(scope="module")
def small():
    return synthetic.small_seir()


@pytest.mark.parametrize("path", ["plain", "batched"])
def test_small_seir_full_size_geometric_matches_oracle(rb, oracle, small, path):
    net = small
    p = dict(net["params"])
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    got = rb.Simulation(g, path=path, **p).run()
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], **_oracle_kw(p, ncls_cap=1))
    np.testing.assert_array_equal(got, want)


def _countdown_params(net):
    """The small SEIR workload in the reference's countdown mode: E, I
    durations equal to the geometric means (48 h, 120 h), R beyond the
    horizon (SIR-like), p = 1 - exp(-2e-5 * 3600) per contact-hour, 1%
    initially infected (the reference's --initial-infected)."""
    return dict(net["params"], transition="countdown", exposed_duration=172800, infectious_duration=432000,
                resistant_duration=100000000, infect_prob=0.069469, initial_infected=0.01, initial_count=0,
                seed=5)


@pytest.mark.parametrize("path", ["auto", "plain", "batched"])
def test_small_seir_full_size_countdown_matches_oracle(rb, oracle, small, path):
    net = small
    p = _countdown_params(net)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    got = rb.Simulation(g, path=path, **p).run()
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], **_oracle_kw(p, ncls_cap=1))
    np.testing.assert_array_equal(got, want)


def test_uneven_batch_sample_matches_oracle(rb, oracle):
    """The uneven batch's smallest, a middle and its largest network (by
    node count), batched, all 1,440 steps, 32 replicas each."""
    batch = synthetic.uneven_batch()
    sizes = np.array([n["n_nodes"] for n in batch["networks"]])
    order = np.argsort(sizes)
    pick = [order[0], order[len(order) // 2], order[-1]]
    nets = [batch["networks"][i] for i in pick]
    assert sizes[pick[0]] < 600 and sizes[pick[-1]] > 45000
    s, e, u, v, n, off = rb.batch_networks(nets)
    p = dict(batch["params"], M=32)
    g = rb.Graph.from_arrays(s, e, u, v, n)
    got = rb.Simulation(g, networks=off, path="batched", **p).run()
    want = oracle.run(s, e, u, v, n, net_first=off, **_oracle_kw(p, ncls_cap=0))
    np.testing.assert_array_equal(got, want)
