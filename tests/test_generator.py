"""The contact_network generator (group model) against the reference's own
generator built from generate_networks/*.c: identical files, byte for byte,
for each of the reference's benchmark scenarios (small populations)."""
import hashlib
import os
import subprocess

import pytest

import replay_b200 as rb

GEN = os.path.join(os.path.dirname(rb.CLI_PATH), "contact_network")

# scenario: (group multiplier, prob_inner, prob_inter), benchmark/benchmark_with_trials.py:12-37
SCENARIOS = {"airport": (0.01, 0.9, 0.5), "villages": (0.1, 0.9, 0.05), "cities": (0.01, 0.9, 0.01),
             "dense": (1.0, 1, 1)}


def scenario_args(name, pop, trial, steps, out):
    mult, p_in, p_out = SCENARIOS[name]
    seed = int(hashlib.sha256(f"{name}_{pop}_{trial}".encode()).hexdigest(), 16) % (10 ** 8)
    return ["2000-01-01T00:00:00", str(steps), "3600", str(pop), str(max(1, int(mult * pop))), str(p_in),
            str(p_out), out, str(seed)]


@pytest.mark.parametrize("name", sorted(SCENARIOS))
@pytest.mark.parametrize("pop", [25, 200])
def test_generator_matches_reference(refshim, tmp_path, name, pop):
    from oracle import ref
    if not os.path.exists(ref.CONTACT_NETWORK_REF):
        pytest.skip("reference generator not built")
    ours, theirs = str(tmp_path / "ours.txt"), str(tmp_path / "ref.txt")
    env = dict(os.environ, TZ="UTC")
    a = subprocess.run([GEN] + scenario_args(name, pop, 1, 6, ours), capture_output=True, text=True, env=env)
    b = subprocess.run([ref.CONTACT_NETWORK_REF] + scenario_args(name, pop, 1, 6, theirs), capture_output=True,
                       text=True, env=env)
    assert a.returncode == 0 and b.returncode == 0
    assert a.stdout.replace(ours, "OUT") == b.stdout.replace(theirs, "OUT")
    with open(ours, "rb") as f1, open(theirs, "rb") as f2:
        assert f1.read() == f2.read()


def test_generated_file_parses(tmp_path):
    out = str(tmp_path / "g.txt")
    subprocess.run([GEN] + scenario_args("villages", 100, 2, 3, out), check=True, capture_output=True,
                   env=dict(os.environ, TZ="UTC"))
    r = rb.parse_contacts(out)
    # the reference parser also reads the NODE_LIST header as a (malformed) contact line
    assert r["n_nodes"] == 100 and r["n_malformed"] == 1 and len(r["start"]) > 0
    assert (r["end"] >= r["start"]).all()
