"""Generates the golden fixtures in tests/golden/ from the reference itself.

Needs the reference built from its own sources (make -C oracle ref, reads
the reference tree).  Every fixture records the reference's output on a small
seeded input:

  parse_cases.json     contact files (text) -> parsed arrays or failure
  windows.npz          NCLS hit lists (with the nbuf = nlists cap), FP32 CSRs
                       (build_csr_from_intervals) at weight scales 1 and 1/3,
                       and Eigen SpMM exposures, for random networks
  replay_*.csv         summary and node-state CSVs of `replay --cpu-only` in
                       deterministic settings (every node infected at t0,
                       infect-prob 1, so rand() never decides an outcome)

Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from replay_b200 import synthetic  # noqa: E402

PARSE_CASES = {
    "basic": "NODE_LIST 1 2 3 4 5\n"
             "1, 2, 1970-01-01T00:00:00Z, 1970-01-01T00:01:00Z; \n"
             "2, 3, 1970-01-01T00:00:30Z, 1970-01-01T00:02:00Z;\n",
    "comments_and_malformed": "NODE_LIST 10 20 30\n"
                              "# a comment line\n"
                              "10, 20, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n"
                              "garbage line\n"
                              "\n"
                              "20, 30, 2000-01-01T00:30:00Z, 2000-01-01T02:00:00Z;\n",
    "normalised_fields": "NODE_LIST 55 63 65 22 23052832\n"
                         "55, 22, 2000-01-01T05:24:44Z, 2000-01-01T25:59:59Z;\n"
                         "22, 23052832, 2000-01-01T09:01:33Z, 2000-01-01T22:34:32Z;\n"
                         "55, 22, 2000-01-05T20:06:55Z, 2001-02-20T21:33:05Z;\n"
                         "63, 65, 2000-13-01T00:00:00Z, 2000-02-30T00:00:60Z;\n",
    "crlf_and_no_semicolon": "NODE_LIST 1 2 3\r\n"
                             "1, 2, 2010-06-01T12:00:00Z, 2010-06-01T12:30:00Z;\r\n"
                             "2, 3, 2010-06-01T12:10:00Z, 2010-06-01T13:00:00Z\r\n",
    "first_appearance_order": "NODE_LIST 7 8 9 4\n"
                              "9, 4, 2000-01-01T00:00:00Z, 2000-01-01T00:10:00Z;\n"
                              "8, 9, 2000-01-01T00:05:00Z, 2000-01-01T00:20:00Z;\n"
                              "7, 4, 2000-01-01T00:07:00Z, 2000-01-01T00:09:00Z;\n",
    "bad_timestamp_skipped": "NODE_LIST 1 2\n"
                             "1, 2, 1969-12-31T23:59:59Z, 1970-01-01T00:10:00Z;\n"
                             "1, 2, notatime, 1970-01-01T00:10:00Z;\n"
                             "1, 2, 1970-01-01T00:00:00Z, 1970-01-01T00:10:00Z;\n",
    "tabs_and_extra": "NODE_LIST\t3\t1\t2\n"
                      "  3,\t1,\t2005-05-05T05:05:05Z ,  2005-05-05T06:05:05Z ; trailing\n"
                      "1, 2, 2005-05-05T05:35:05, 2005-05-05T05:45:05;\n",
    "self_loop": "NODE_LIST 1 2\n"
                 "1, 1, 2000-01-01T00:00:00Z, 2000-01-01T00:30:00Z;\n"
                 "1, 2, 2000-01-01T00:00:00Z, 2000-01-01T00:30:00Z;\n",
    "bad_header": "NODE 1 2 3\n1, 2, 2000-01-01T00:00:00Z, 2000-01-01T00:10:00Z;\n",
    "duplicate_id": "NODE_LIST 1 2 2\n1, 2, 2000-01-01T00:00:00Z, 2000-01-01T00:10:00Z;\n",
    "negative_id": "NODE_LIST 1 -2\n1, 2, 2000-01-01T00:00:00Z, 2000-01-01T00:10:00Z;\n",
    "no_edges": "NODE_LIST 1 2\n# nothing\n",
    "spaces_before_commas_fatal": "NODE_LIST 1 2\n"
                                  "1 , 2 , 2000-01-01T00:00:00Z , 2000-01-01T00:10:00Z ;\n",
}


def parse_fixtures():
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name, text in PARSE_CASES.items():
            path = os.path.join(td, name + ".txt")
            with open(path, "w", newline="") as f:
                f.write(text)
            r = ref.parse(path)
            if r["error"] or len(r["start"]) == 0:
                out[name] = {"text": text, "ok": False}
            else:
                out[name] = {"text": text, "ok": True, "n_nodes": r["n_nodes"],
                             "start": r["start"].tolist(), "end": r["end"].tolist(),
                             "u": r["u"].tolist(), "v": r["v"].tolist()}
    # The reference exits from inside its parser when more lines parse than
    # were counted; the shim cannot run that case, so it is recorded as failing.
    out["spaces_before_commas_fatal"]["ok"] = False
    with open(os.path.join(HERE, "parse_cases.json"), "w") as f:
        json.dump(out, f, indent=1)


def window_fixtures():
    arrays = {}
    cases = []
    for seed in range(6):
        net = synthetic.tiny(seed=100 + seed, n_nodes=25, n_contacts=120, span=4 * 3600, max_dur=3000,
                             negative=(seed % 3 == 2))
        s, e, u, v = net["start"], net["end"], net["u"], net["v"]
        rng = np.random.default_rng(seed)
        for k in range(8):
            W = int(rng.choice([300, 900, 3600]))
            ws = int(net["t0"] + rng.integers(-W, 4 * 3600))
            q = ref.window_query(s, e, u, v, ws, ws + W)
            tag = f"s{seed}_w{k}"
            for scale_name, scale in (("1", 1.0), ("third", np.float32(1 / 3))):
                rp, col, val = ref.build_csr(q["start"], q["end"], q["u"], q["v"], net["n_nodes"], ws, ws + W,
                                             np.float32(scale))
                m = 3
                b = (rng.random(net["n_nodes"] * m) < 0.4).astype(np.float32)
                c = ref.cpu_spmm(rp, col, val, net["n_nodes"], b, m)
                arrays[f"{tag}_{scale_name}_rp"] = rp
                arrays[f"{tag}_{scale_name}_col"] = col
                arrays[f"{tag}_{scale_name}_val"] = val
                arrays[f"{tag}_{scale_name}_b"] = b
                arrays[f"{tag}_{scale_name}_c"] = c
            arrays[f"{tag}_hit_u"] = q["u"]
            arrays[f"{tag}_hit_v"] = q["v"]
            arrays[f"{tag}_hit_start"] = q["start"]
            cases.append({"tag": tag, "seed": 100 + seed, "negative": bool(seed % 3 == 2), "ws": ws, "we": ws + W,
                          "nlists": q["nlists"]})
    np.savez_compressed(os.path.join(HERE, "windows.npz"), **arrays)
    with open(os.path.join(HERE, "windows.json"), "w") as f:
        json.dump(cases, f, indent=1)


REPLAY_CASES = {
    # every node infected at t0 (p0 = 1), infect-prob 1: deterministic SEIRS
    "seirs": ["--M", 3, "--iterations", 40, "--step-size", 900, "--static-network-duration", 900,
              "--initial-infected", 1.0, "--infect-prob", 1.0, "--exposed-duration", 1800,
              "--infectious-duration", 2700, "--resistant-duration", 3600],
    "sis_fractional_step": ["--M", 2, "--iterations", 30, "--step-size", 1000.5, "--static-network-duration", 3000,
                            "--initial-infected", 1.0, "--infect-prob", 1.0, "--exposed-duration", 0,
                            "--infectious-duration", 4000, "--resistant-duration", 0],
    "no_infection": ["--M", 2, "--iterations", 10, "--initial-infected", 0.0, "--infect-prob", 0.5,
                     "--exposed-duration", 3600, "--infectious-duration", 3600, "--resistant-duration", 3600],
}


def replay_fixtures():
    net = synthetic.tiny(seed=7, n_nodes=30, n_contacts=600, span=12 * 3600, max_dur=4000)
    graph = os.path.join(HERE, "replay_graph.txt")
    synthetic.write_contact_file(graph, net)
    meta = {}
    for name, args in REPLAY_CASES.items():
        out = os.path.join(HERE, f"replay_{name}.csv")
        nodes = os.path.join(HERE, f"replay_{name}_nodes.csv")
        full = [graph, "--cpu-only", "-q", "--start-time", net["t0"], "--summary-out", out,
                "--node-state-out", nodes] + args
        r = ref.run_cli(full)
        assert r.returncode == 0, r.stderr
        meta[name] = [str(a) for a in args] + ["--start-time", str(net["t0"])]
    with open(os.path.join(HERE, "replay_cases.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    if not ref.available():
        sys.exit("reference not built: make -C oracle ref")
    parse_fixtures()
    window_fixtures()
    replay_fixtures()
    print("golden fixtures written to", HERE)
