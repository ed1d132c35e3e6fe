"""Host-side product code that runs without a GPU: the C ABI's exports and
argument checks, the multithreaded contact-file parser, and the CLI's
error exits.  The parser is compared with the golden fixtures (generated
by the reference) and with the C oracle on randomised files."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import replay_b200 as rb
from replay_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "replay.h")


def declared_symbols():
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"RP_API\s+[\w\s\*]+?\b(rp_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    L = rb.lib()
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"
    assert set(_lib.SIGNATURES) <= set(names)
    assert rb.version().startswith("replay-b200")


def test_bad_arguments_fail_with_status_before_any_device_work():
    L = rb.lib()
    import ctypes as C
    h = C.c_void_p()
    s = np.array([0, 10], np.int64)
    e = np.array([5, 20], np.int64)
    u = np.array([0, 1], np.int32)
    v = np.array([1, 7], np.int32)  # node 7 outside [0, 3)
    st = L.rp_graph_from_arrays(s.ctypes.data, e.ctypes.data, u.ctypes.data, v.ctypes.data, 2, 3, 0, C.byref(h))
    assert st == 1 and b"outside" in L.rp_last_error()
    assert L.rp_sim_create(None, None, C.byref(h)) == 1
    with pytest.raises(rb.ReplayError):
        rb.parse_contacts("/nonexistent/contacts.txt")


def _write(tmp_path, name, text):
    p = tmp_path / (name + ".txt")
    with open(p, "w", newline="") as f:
        f.write(text)
    return str(p)


def test_parser_matches_reference_fixtures(golden_dir, tmp_path):
    with open(os.path.join(golden_dir, "parse_cases.json")) as f:
        cases = json.load(f)
    for name, case in cases.items():
        path = _write(tmp_path, name, case["text"])
        if not case["ok"]:
            try:
                n = len(rb.parse_contacts(path)["start"])
            except rb.ReplayError:
                n = 0
            assert n == 0, name
            continue
        r = rb.parse_contacts(path)
        assert r["n_nodes"] == case["n_nodes"], name
        for k in ("start", "end", "u", "v"):
            np.testing.assert_array_equal(r[k], np.array(case[k]), err_msg=f"{name}:{k}")


def random_contact_text(rng, n_lines, n_ids=40):
    ids = rng.choice(10**7, n_ids, replace=False)
    out = ["NODE_LIST " + " ".join(str(i) for i in ids) + ("\r\n" if rng.random() < 0.3 else "\n")]
    for k in range(n_lines):
        r = rng.random()
        if r < 0.03:
            out.append("# comment %d\n" % k)
            continue
        if r < 0.05:
            out.append("not a contact line\n")
            continue
        if r < 0.06:
            out.append("\n")
            continue
        a, b = rng.choice(ids, 2)
        y = int(rng.integers(1999, 2003))
        mo, d, h, mi, sec = (int(rng.integers(1, 13)), int(rng.integers(1, 29)), int(rng.integers(0, 24)),
                             int(rng.integers(0, 60)), int(rng.integers(0, 60)))
        if rng.random() < 0.05:  # out-of-range fields are normalised by timegm
            h, sec = 25, 61
        t0 = f"{y:04d}-{mo:02d}-{d:02d}T{h:02d}:{mi:02d}:{sec:02d}Z"
        t1 = f"{y:04d}-{mo:02d}-{d:02d}T{min(h + 1, 23):02d}:{mi:02d}:{sec:02d}Z"
        sep = rng.choice([", ", ",", ",\t", ",  "])
        end = rng.choice([";\n", ";\r\n", "; trailing\n", ";\n"])
        out.append(f"{a}{sep}{b}{sep}{t0}{sep}{t1}{end}")
    return "".join(out)


@pytest.mark.parametrize("seed,n_lines", [(0, 50), (1, 2000), (2, 40000)])
def test_parser_matches_oracle_on_random_files(oracle, tmp_path, seed, n_lines):
    rng = np.random.default_rng(seed)
    path = _write(tmp_path, f"r{seed}", random_contact_text(rng, n_lines))
    got = rb.parse_contacts(path)
    want = oracle.parse_file(path)
    assert want["error"] == 0
    assert got["n_nodes"] == want["n_nodes"] and got["n_index"] == want["n_index"]
    assert got["n_malformed"] == want["n_malformed"]
    for k in ("start", "end", "u", "v"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_parser_first_appearance_across_threads(oracle, tmp_path):
    """The parser reads a large file in parallel ranges and numbers nodes
    by first appearance over the whole file.  Here new ids keep appearing
    down to the last lines (some first as the second endpoint), and lines
    whose timestamp is rejected (-1, 1969-12-31T23:59:59Z) name ids that no
    other line does: those must get no number."""
    rng = np.random.default_rng(11)
    n_lines, n_ids = 60000, 6000
    ids = rng.permutation(n_ids) * 7 + 3
    rejected = np.arange(n_ids, n_ids + 300) * 7 + 3
    out = ["NODE_LIST " + " ".join(str(int(x)) for x in np.concatenate([ids, rejected])) + "\n"]
    k_rej = 0
    for k in range(n_lines):
        pool = ids[: 2 + (k * n_ids) // n_lines]
        if k % 200 == 7:
            out.append(f"{rejected[k_rej]}, {pool[0]}, 1969-12-31T23:59:59Z, 2000-01-01T00:00:00Z;\n")
            k_rej += 1
            continue
        a = int(rng.choice(pool[:-1]))
        b = int(pool[-1]) if rng.random() < 0.3 else int(rng.choice(pool))
        if a == b:
            b = int(pool[0]) if a != pool[0] else int(pool[1])
        t0 = 946684800 + int(rng.integers(0, 86400 * 20))
        s = np.datetime64(t0, "s").astype(str) + "Z"
        e = np.datetime64(t0 + int(rng.integers(1, 3600)), "s").astype(str) + "Z"
        out.append(f"{a}, {b}, {s}, {e};\n")
    text = "".join(out)
    assert len(text) > 2 << 20
    path = _write(tmp_path, "order", text)
    got = rb.parse_contacts(path)
    want = oracle.parse_file(path)
    assert want["error"] == 0
    assert got["n_index"] == want["n_index"]
    assert want["n_index"] > n_ids - 100  # nearly every id is used
    assert got["n_malformed"] == want["n_malformed"]
    for k in ("start", "end", "u", "v"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def _fixed_form_text():
    lines = [
        "1, 2, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",
        "123456789, 2, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",  # 9-digit id, not listed
        "1234567890, 2, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",  # 10 digits: general rules
        "3, 4, 2000-13-40T25:61:61Z, 2001-02-30T00:00:00Z;\r\n",  # normalised like timegm
        "5, 6, 1969-12-31T23:59:59Z, 2000-01-01T00:00:00Z;\n",  # start == -1: rejected
        "# 7, 8, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",
        "7,8, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",  # one separator without blank
        "9, 10, 2000-01-01T00:00:00, 2000-01-01T01:00:00Z;\n",  # no Z on the start
        "11, 12, 2000-1-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",  # short month field
        " 13, 14, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;\n",  # leading blank
        "15, 16, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z; trailing\n",
        "17, 18, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;" + "x" * 150000 + "\n",  # > one chunk
        "19, 20, 2000-01-01T00:00:00Z, 2000-01-01T01:00:00Z;",  # no final newline
    ]
    ids = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 123456789, 1234567890]
    return "NODE_LIST " + " ".join(map(str, ids)) + "\n" + "".join(lines)


def test_parser_fixed_form_lines_match_reference(refshim, tmp_path):
    path = _write(tmp_path, "fixed_ref", _fixed_form_text())
    got = rb.parse_contacts(path)
    want = refshim.parse(path)
    for k in ("start", "end", "u", "v"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def test_parser_fixed_form_lines_and_their_edges(oracle, tmp_path):
    """Lines in the generator's exact form take a fixed-offset path; lines
    that only nearly have that form, and a fixed-form line longer than one
    fgets chunk (whose tail the reference reads as further lines), must
    come out as the general rules read them."""
    path = _write(tmp_path, "fixed", _fixed_form_text())
    got = rb.parse_contacts(path)
    want = oracle.parse_file(path)
    assert want["error"] == 0
    assert got["n_index"] == want["n_index"] and got["n_malformed"] == want["n_malformed"]
    for k in ("start", "end", "u", "v"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    assert len(got["start"]) >= 10


def test_parser_matches_reference_on_random_files(refshim, tmp_path):
    rng = np.random.default_rng(7)
    path = _write(tmp_path, "ref", random_contact_text(rng, 3000))
    got = rb.parse_contacts(path)
    want = refshim.parse(path)
    assert got["n_nodes"] == want["n_nodes"]
    for k in ("start", "end", "u", "v"):
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


def run_cli(args):
    return subprocess.run([rb.CLI_PATH] + [str(a) for a in args], capture_output=True, text=True, timeout=60)


def test_cli_error_exits(tmp_path):
    assert run_cli([]).returncode == 1
    assert run_cli([str(tmp_path / "missing.txt")]).returncode == 1
    good = _write(tmp_path, "g", "NODE_LIST 1 2\n1, 2, 2000-01-01T00:00:00Z, 2000-01-01T00:10:00Z;\n")
    assert run_cli([good, "--no-such-flag", "1"]).returncode == 1
    assert run_cli([good, "--M"]).returncode == 1
    assert run_cli([good, "--transition", "sideways"]).returncode == 1
