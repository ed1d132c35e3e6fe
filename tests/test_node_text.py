"""Node-state CSV text formatted on the GPU (rp_sim_run_text): the CLI's
--node-state-out output is byte-identical to the reference's on the golden
runs, and the device text equals the host formatting of the node states
over multi-chunk steps."""
import json
import os
import subprocess

import numpy as np
import pytest

from replay_b200 import synthetic

pytestmark = pytest.mark.gpu

STATE_NAMES = ["susceptible", "incubating", "infectious", "resistant"]


@pytest.fixture(scope="module")
def rb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import replay_b200
    replay_b200.lib()
    return replay_b200


@pytest.mark.parametrize("name", ["seirs", "sis_fractional_step", "no_infection"])
def test_cli_node_state_csv_matches_reference(rb, golden_dir, tmp_path, name):
    with open(os.path.join(golden_dir, "replay_cases.json")) as f:
        args = json.load(f)[name]
    nodes, summary = str(tmp_path / "nodes.csv"), str(tmp_path / "summary.csv")
    cmd = [rb.CLI_PATH, os.path.join(golden_dir, "replay_graph.txt"), "-q", "--summary-out", summary,
           "--node-state-out", nodes] + args
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    for got, want in ((nodes, f"replay_{name}_nodes.csv"), (summary, f"replay_{name}.csv")):
        with open(got, "rb") as a, open(os.path.join(golden_dir, want), "rb") as b:
            assert a.read() == b.read(), want


def test_device_text_equals_host_formatting_across_chunks(rb):
    net = synthetic.tiny(seed=91, n_nodes=2000, n_contacts=20000, span=4 * 3600)
    g = rb.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"])
    kw = dict(M=700, iterations=3, step_size=1800.0, window=1800, start_time=net["t0"], seed=2,
              transition="geometric", beta=8e-4, p_ei=0.3, p_ir=0.2, initial_count=40, record_node_states=True)
    states, times = [], []
    want_counts = rb.Simulation(g, **kw).run(node_states=lambda k, ts, st: states.append(st) or times.append(ts))
    chunks = {}
    got_counts = rb.Simulation(g, **kw).run_text(lambda k, ts, data: chunks.setdefault(k, []).append(data) and 0)
    np.testing.assert_array_equal(got_counts, want_counts)
    assert len(chunks) == 4 and all(len(v) >= 2 for v in chunks.values())  # 700 replicas span 2 chunks
    for k, (st, ts) in enumerate(zip(states, times)):
        want = "".join(f"{ts},{r},{i},{STATE_NAMES[s]}\n" for r in range(st.shape[0]) for i, s in enumerate(st[r]))
        assert b"".join(chunks[k]).decode() == want
