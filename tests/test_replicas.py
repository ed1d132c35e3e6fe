"""Replica sharding: shards with a replica offset reproduce the unsharded
run, on the CPU oracle across two gloo ranks and on the GPU."""
import os

import numpy as np
import pytest

from replay_b200 import synthetic
from replay_b200.replicas import shard


def test_shard_covers_replicas_in_whole_words():
    for m in (1, 31, 32, 33, 100, 128, 4096, 4100):
        for world in (1, 2, 3, 8):
            parts = [shard(m, world, r) for r in range(world)]
            assert sum(c for _, c in parts) == m
            pos = 0
            for off, cnt in parts:
                assert off == pos and off % 32 == 0 or cnt == 0
                pos += cnt


KW = dict(n_steps=16, step_size=1800.0, window=1800, transition=1, seed=9, beta=8e-4, p_ei=0.3, p_ir=0.2,
          p_rs=0.05, initial_count=3)


def _gloo_rank(rank, world, port, path):
    import torch.distributed as dist

    from oracle import orc
    from replay_b200.replicas import gather_counts
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net = synthetic.tiny(seed=80, n_nodes=60, n_contacts=900)
        m = 100
        off, cnt = shard(m, world, rank)
        local = orc.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], n_replicas=cnt,
                        replica_offset=off, start_time=net["t0"], **KW)
        full = gather_counts(local, m)
        if rank == 0:
            np.save(path, full)
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_reproduce_unsharded_oracle_run(oracle, tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    path = str(tmp_path / "gathered.npy")
    mp.spawn(_gloo_rank, args=(2, port, path), nprocs=2, join=True)
    net = synthetic.tiny(seed=80, n_nodes=60, n_contacts=900)
    want = oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], n_replicas=100,
                      start_time=net["t0"], **KW)
    np.testing.assert_array_equal(np.load(path), want)


@pytest.mark.gpu
@pytest.mark.parametrize("path,transition", [("batched", "geometric"), ("plain", "geometric"),
                                             ("plain", "countdown")])
def test_gpu_shards_reproduce_unsharded_run(oracle, path, transition):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200 as rb
    net = synthetic.tiny(seed=81, n_nodes=90, n_contacts=1800)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    kw = dict(iterations=20, step_size=1800.0, window=1800, start_time=net["t0"], seed=4, transition=transition,
              path=path, initial_count=4)
    if transition == "geometric":
        kw.update(beta=9e-4, p_ei=0.3, p_ir=0.15)
    else:
        kw.update(infect_prob=0.4, exposed_duration=3600, infectious_duration=7200, resistant_duration=3600)
    m = 100
    full = rb.Simulation(g, M=m, **kw).run()
    parts = [rb.Simulation(g, M=cnt, replica_offset=off, **kw).run() for off, cnt in (shard(m, 3, r) for r in range(3))]
    np.testing.assert_array_equal(np.concatenate(parts, axis=1), full)
    okw = dict(n_replicas=m, n_steps=20, step_size=1800.0, window=1800, start_time=net["t0"], seed=4,
               initial_count=4, transition=0 if transition == "countdown" else 1,
               **{k: v for k, v in kw.items() if k in ("beta", "p_ei", "p_ir", "infect_prob", "exposed_duration",
                                                       "infectious_duration", "resistant_duration")})
    np.testing.assert_array_equal(full, oracle.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], **okw))
