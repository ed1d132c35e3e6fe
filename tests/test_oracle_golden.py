"""Pins the CPU oracle against golden vectors produced by the reference.

Fixtures under tests/golden/ were generated by make_golden.py from the
reference built from its own sources (parser, NCLS window query with its
hit cap, build_csr_from_intervals, the Eigen CPU SpMM, and the `replay
--cpu-only` summary CSV in settings where no random draw decides an
outcome).  These run without a GPU.
"""
import json
import math
import os
import struct

import numpy as np
import pytest

from replay_b200 import synthetic


def _write(tmp_path, name, text):
    p = tmp_path / (name + ".txt")
    with open(p, "w", newline="") as f:
        f.write(text)
    return str(p)


def test_philox4x32_10_known_answers(oracle):
    # Known-answer vectors published with Random123 (Salmon et al., SC'11).
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in cases:
        assert oracle.philox(ctr, key) == want


def _infection_uniform(oracle, seed, node, step, r):
    """The 64-bit geometric-mode infection uniform of replica r, restated
    from the stream layout: top 8 bits bit-sliced (bit r % 32 of the outputs
    of counters (node, step, r / 32, 4 | j << 4), j = 0, 1), low 56 bits the
    top 56 of outputs 0-1 of counter (node, step, r, 12)."""
    key = [seed & 0xFFFFFFFF, seed >> 32]
    u8 = 0
    for j in range(2):
        for x in oracle.philox([node, step, r >> 5, 4 | j << 4], key):
            u8 = u8 << 1 | (x >> (r & 31)) & 1
    x = oracle.philox([node, step, r, 12], key)
    return u8 << 56 | (x[0] << 32 | x[1]) >> 8


def test_infection_uniform_layout_and_rate(oracle):
    rng = np.random.default_rng(3)
    seed = 0x1234_5678_9ABC_DEF0
    for _ in range(300):
        node, step, r = (int(v) for v in rng.integers(0, 2**31, 3))
        U = _infection_uniform(oracle, seed, node, step, r)
        # thresholds just around U: the top byte ties, the tail decides
        for P in (np.nextafter(np.float32(U / 2**64), np.float32(2)),
                  np.nextafter(np.float32(U / 2**64), np.float32(0)), np.float32(rng.random())):
            P = float(P)
            if not 0.0 < P < 1.0:
                continue
            assert oracle.infect_event(seed, node, step, r, P) == (U < int(math.ldexp(P, 64))), (node, r, P)
    assert oracle.infect_event(seed, 1, 2, 3, 1.0) and not oracle.infect_event(seed, 1, 2, 3, 0.0)
    assert not oracle.infect_event(seed, 1, 2, 3, float("nan"))
    # event rates, for a P just above a top-byte boundary and a generic one
    n = 20000
    for P in (np.float32(3 / 256 + 1e-5), np.float32(0.3)):
        hits = sum(oracle.infect_event(seed, 7 + i // 4096, 11, i % 4096, float(P)) for i in range(n))
        assert abs(hits / n - P) < 5 * math.sqrt(P * (1 - P) / n), (P, hits / n)


def _flow_uniform(oracle, seed, node, step, r):
    """The 64-bit flow uniform of replica r, restated from the stream
    layout: bit k (k = 0 is 2^-1) is bit r % 32 of output k % 4 of counter
    (node, step, r / 32, (k / 4) << 4)."""
    key = [seed & 0xFFFFFFFF, seed >> 32]
    u = 0
    for j in range(16):
        for x in oracle.philox([node, step, r >> 5, j << 4], key):
            u = u << 1 | (x >> (r & 31)) & 1
    return u


def test_flow_uniform_layout_and_rate(oracle):
    rng = np.random.default_rng(4)
    seed = 0x0FED_CBA9_8765_4321
    for _ in range(200):
        node, step, r = (int(v) for v in rng.integers(0, 2**31, 3))
        U = _flow_uniform(oracle, seed, node, step, r)
        for p in (np.nextafter(np.float32(U / 2**64), np.float32(2)),
                  np.nextafter(np.float32(U / 2**64), np.float32(0)), np.float32(rng.random())):
            T, always = oracle.flow_threshold(float(p))
            if always or T == 0:
                continue
            assert T == int(math.ldexp(float(p), 64))
            assert oracle.flow_event(seed, node, step, r, float(p)) == (U < T), (node, r, p)
    assert oracle.flow_threshold(1.0) == (0, True) and oracle.flow_event(seed, 1, 2, 3, 1.0)
    assert oracle.flow_threshold(0.0) == (0, False) and not oracle.flow_event(seed, 1, 2, 3, 0.0)
    n = 20000
    for p in (np.float32(1 / 48), np.float32(0.5)):
        hits = sum(oracle.flow_event(seed, 5 + i // 4096, 9, i % 4096, float(p)) for i in range(n))
        assert abs(hits / n - p) < 5 * math.sqrt(p * (1 - p) / n), (p, hits / n)


def _f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def test_one_minus_exp_neg_accuracy_and_bound(oracle):
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.float32(10.0) ** rng.uniform(-12, 1.5, 4000),
                         np.array([0.0, 1e-30, 1e-8, 0.5, 1.0, 2.0, 20.0, 88.0], np.float32)]).astype(np.float32)
    for x in xs:
        x = float(x)
        got = oracle.one_minus_exp_neg(x)
        want = -math.expm1(-x)
        assert abs(got - want) <= 2.5 * np.spacing(np.float32(want)) + 1e-45, (x, got, want)
        # P <= x: the bound the batched kernel uses to skip exact evaluation
        assert got <= _f32(x)


def test_parse_matches_reference_fixtures(oracle, golden_dir, tmp_path):
    with open(os.path.join(golden_dir, "parse_cases.json")) as f:
        cases = json.load(f)
    for name, case in cases.items():
        r = oracle.parse_file(_write(tmp_path, name, case["text"]))
        if not case["ok"]:
            assert r["error"] != 0 or len(r.get("start", [])) == 0, name
            continue
        assert r["error"] == 0, name
        assert r["n_nodes"] == case["n_nodes"], name
        for k in ("start", "end", "u", "v"):
            np.testing.assert_array_equal(r[k], np.array(case[k]), err_msg=f"{name}:{k}")


def _window_net(case):
    return synthetic.tiny(seed=case["seed"], n_nodes=25, n_contacts=120, span=4 * 3600, max_dur=3000,
                          negative=case["negative"])


def test_window_query_csr_and_spmm_match_reference_fixtures(oracle, golden_dir):
    with open(os.path.join(golden_dir, "windows.json")) as f:
        cases = json.load(f)
    z = np.load(os.path.join(golden_dir, "windows.npz"))
    assert len(cases) == 48
    for case in cases:
        net = _window_net(case)
        tag, ws, we = case["tag"], case["ws"], case["we"]
        ss, se, su, sv, perm, nl = oracle.sorted_index(net["start"], net["end"], net["u"], net["v"])
        assert nl == case["nlists"], tag
        hits = oracle.window_hits(ss, se, nl, ws, we)
        np.testing.assert_array_equal(su[hits], z[f"{tag}_hit_u"], err_msg=tag)
        np.testing.assert_array_equal(sv[hits], z[f"{tag}_hit_v"], err_msg=tag)
        hs = [oracle.hit_coords(ss[h], se[h], ws)[0] for h in hits]
        np.testing.assert_array_equal(np.array(hs, np.int64).reshape(-1), z[f"{tag}_hit_start"], err_msg=tag)
        for scale_name, scale in (("1", np.float32(1.0)), ("third", np.float32(1 / 3))):
            rp, col, val = oracle.csr_f32(ss, se, su, sv, hits, net["n_nodes"], ws, we, scale)
            key = f"{tag}_{scale_name}"
            np.testing.assert_array_equal(rp, z[key + "_rp"], err_msg=key)
            np.testing.assert_array_equal(col, z[key + "_col"], err_msg=key)
            np.testing.assert_array_equal(val.view(np.int32), z[key + "_val"].view(np.int32), err_msg=key)
            c = oracle.spmm_f32(rp, col, val, net["n_nodes"], z[key + "_b"], 3)
            np.testing.assert_array_equal(c.view(np.int32), z[key + "_c"].view(np.int32), err_msg=key)


FLAG_TO_PARAM = {"--M": ("n_replicas", int), "--iterations": ("n_steps", int), "--step-size": ("step_size", float),
                 "--static-network-duration": ("window", int), "--initial-infected": ("initial_infected", float),
                 "--infect-prob": ("infect_prob", float), "--exposed-duration": ("exposed_duration", int),
                 "--infectious-duration": ("infectious_duration", int),
                 "--resistant-duration": ("resistant_duration", int), "--start-time": ("start_time", int)}


def cli_args_to_params(args):
    kw = {}
    for flag, val in zip(args[::2], args[1::2]):
        name, conv = FLAG_TO_PARAM[flag]
        kw[name] = conv(val)
    return kw


def read_summary_csv(path):
    with open(path) as f:
        header = f.readline().strip()
        rows = np.array([[int(x) for x in line.split(",")] for line in f if line.strip()], np.int64)
    assert header == "time,simulation_id,exposed,infectious,resistant,susceptible"
    return rows


@pytest.mark.parametrize("name", ["seirs", "sis_fractional_step", "no_infection"])
def test_countdown_replay_matches_reference_csv(oracle, golden_dir, name):
    with open(os.path.join(golden_dir, "replay_cases.json")) as f:
        args = json.load(f)[name]
    kw = cli_args_to_params(args)
    got = oracle.parse_file(os.path.join(golden_dir, "replay_graph.txt"))
    counts = oracle.run(got["start"], got["end"], got["u"], got["v"], got["n_nodes"], transition=0, seed=5, **kw)
    rows = read_summary_csv(os.path.join(golden_dir, f"replay_{name}.csv"))
    T, M = kw["n_steps"], kw["n_replicas"]
    assert rows.shape == ((T + 1) * M, 6)
    np.testing.assert_array_equal(rows[:, 2:].reshape(T + 1, M, 4), counts)
    np.testing.assert_array_equal(rows[:, 1].reshape(T + 1, M), np.tile(np.arange(M), (T + 1, 1)))
    ws, we, sc, ts = oracle.schedule(kw["start_time"], kw.get("step_size", 3600.0), kw.get("window", 3600), T)
    times = np.concatenate([[kw["start_time"]], ts])
    np.testing.assert_array_equal(rows[:, 0].reshape(T + 1, M), np.repeat(times[:, None], M, axis=1))


def test_window_hits_half_open(oracle, tmp_path):
    # Half-open overlap (start < we && ws < end, intervaldb.h:188-189):
    # a contact ending exactly at a window start is not a hit.
    text = ("NODE_LIST 1 2 3 4\n"
            "1, 2, 1970-01-01T00:00:10Z, 1970-01-01T00:00:20Z;\n"
            "2, 3, 1970-01-01T00:00:50Z, 1970-01-01T00:01:10Z;\n"
            "3, 4, 1970-01-01T00:02:00Z, 1970-01-01T00:03:00Z;\n"
            "1, 4, 1970-01-01T00:00:00Z, 1970-01-01T00:04:00Z;\n")
    r = oracle.parse_file(_write(tmp_path, "g", text))
    ss, se, su, sv, perm, nl = oracle.sorted_index(r["start"], r["end"], r["u"], r["v"])
    counts = [len(oracle.window_hits(ss, se, len(ss), 60 * k, 60 * (k + 1))) for k in range(4)]
    assert counts == [3, 2, 2, 1]


STATE_NAMES = ["susceptible", "incubating", "infectious", "resistant"]


def format_node_rows(states, times):
    """Reference node-CSV lines of (T+1, M, N) states (replicas outer)."""
    out = ["time,simulation_id,node_id,state\n"]
    for t, ts in enumerate(times):
        for r in range(states.shape[1]):
            out.extend(f"{ts},{r},{i},{STATE_NAMES[s]}\n" for i, s in enumerate(states[t, r]))
    return "".join(out)


@pytest.mark.parametrize("name", ["seirs", "sis_fractional_step", "no_infection"])
def test_countdown_node_states_match_reference_csv(oracle, golden_dir, name):
    with open(os.path.join(golden_dir, "replay_cases.json")) as f:
        kw = cli_args_to_params(json.load(f)[name])
    got = oracle.parse_file(os.path.join(golden_dir, "replay_graph.txt"))
    _, states = oracle.run(got["start"], got["end"], got["u"], got["v"], got["n_nodes"], transition=0, seed=5,
                           node_states=True, **kw)
    T = kw["n_steps"]
    ws, we, sc, ts = oracle.schedule(kw["start_time"], kw.get("step_size", 3600.0), kw.get("window", 3600), T)
    text = format_node_rows(states, [kw["start_time"]] + list(ts))
    with open(os.path.join(golden_dir, f"replay_{name}_nodes.csv")) as f:
        assert text == f.read()
