"""Closing a graph or simulation keeps its device blocks for the next one
(rp_release_cached_memory returns them): a second create/run/close cycle of
the same shapes reuses the kept blocks without growing device memory, gives
the same counts, and releasing the cache gives the memory back."""
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


def _cycle(rb, net, p):
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    s = rb.Simulation(g, path="batched", csr="per-step", **p)
    counts = s.run()
    s.close()
    g.close()
    return counts


def test_closed_handles_keep_blocks_for_the_next(rb):
    import torch
    net = synthetic.dense_stress(seed=8, n_contacts=2_000_000, days=1, steps=96, replicas=1024)
    p = dict(net["params"], M=1024, iterations=24, initial_count=20, seed=3)
    rb.release_cached_memory()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    a = _cycle(rb, net, p)
    free1 = torch.cuda.mem_get_info()[0]
    # the index alone holds 64 MB of contacts, its build more scratch
    assert free0 - free1 > 64 << 20
    b = _cycle(rb, net, p)
    free2 = torch.cuda.mem_get_info()[0]
    np.testing.assert_array_equal(a, b)
    assert free2 >= free1 - (4 << 20)  # the second cycle ran on the kept blocks
    rb.release_cached_memory()
    free3 = torch.cuda.mem_get_info()[0]
    assert free3 - free2 > 64 << 20
    assert abs(free3 - free0) <= 16 << 20
