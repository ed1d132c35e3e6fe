"""The C oracle against the reference's own functions, compiled from its
sources into oracle/_ref/libref_shim.so (skipped where that is not built).

Randomised networks, including negative times (the interval database's
mirrored storage), exercise the NCLS query with its hit cap, the FP32 CSR
builder, the SpMM, the countdown classification behind the CSVs, and the
infection probability (which the oracle evaluates with its own correctly
specified 1 - exp(-x); it must stay within 1e-6 of the reference's expf).
"""
import numpy as np
import pytest

from replay_b200 import synthetic


@pytest.mark.parametrize("seed", range(6))
def test_windows_match_reference(oracle, refshim, seed):
    net = synthetic.tiny(seed=200 + seed, n_nodes=40, n_contacts=400, span=6 * 3600, max_dur=5000,
                         negative=(seed % 2 == 1))
    s, e, u, v, n = net["start"], net["end"], net["u"], net["v"], net["n_nodes"]
    ss, se, su, sv, perm, nl = oracle.sorted_index(s, e, u, v)
    rng = np.random.default_rng(seed)
    for k in range(60):
        W = int(rng.choice([60, 600, 1800, 3600, 7200]))
        ws = int(net["t0"] + rng.integers(-2 * W, 6 * 3600 + W))
        q = refshim.window_query(s, e, u, v, ws, ws + W)
        assert q["nlists"] == nl
        hits = oracle.window_hits(ss, se, nl, ws, ws + W)
        np.testing.assert_array_equal(su[hits], q["u"])
        np.testing.assert_array_equal(sv[hits], q["v"])
        scale = np.float32(1.0 / rng.integers(1, 5))
        rp, col, val = oracle.csr_f32(ss, se, su, sv, hits, n, ws, ws + W, scale)
        rrp, rcol, rval = refshim.build_csr(q["start"], q["end"], q["u"], q["v"], n, ws, ws + W, scale)
        np.testing.assert_array_equal(rp, rrp)
        np.testing.assert_array_equal(col, rcol)
        np.testing.assert_array_equal(val.view(np.int32), rval.view(np.int32))
        b = (rng.random(n * 4) < 0.3).astype(np.float32)
        np.testing.assert_array_equal(oracle.spmm_f32(rp, col, val, n, b, 4).view(np.int32),
                                      refshim.cpu_spmm(rrp, rcol, rval, n, b, 4).view(np.int32))


def test_infection_probability_within_1e6_of_reference(oracle, refshim):
    L = refshim.lib()
    rng = np.random.default_rng(3)
    for p in (1e-4, 0.0695, 0.3, 0.9, 0.999):
        n, m = 512, 4
        expo = np.concatenate([rng.integers(0, 4000, n * m // 2), rng.integers(0, 10 ** 6, n * m // 2)]).astype(
            np.float32)
        cd = np.zeros(n * m, np.int32)
        L.ref_set_durations(3600, 3600, 3600, np.float32(p))
        ref_p = expo.copy()
        L.ref_infection_prob(ref_p, cd, n, m, np.float32(3600.0))
        nlb = -np.log(np.float32(1.0) - np.float32(p)).astype(np.float32)
        # the oracle evaluates 1 - exp(-(-log(1-p)) * e) with e in contact-hours
        ours = np.array([oracle.one_minus_exp_neg(np.float32(nlb * np.float32(x / 3600.0))) for x in expo],
                        np.float32)
        assert np.max(np.abs(ours.astype(np.float64) - ref_p.astype(np.float64))) <= 1e-6, p


def test_countdown_classification_matches_reference_csv(oracle, refshim, tmp_path):
    L = refshim.lib()
    Ed, Id, Rd = 1800, 2700, 3600
    L.ref_set_durations(Ed, Id, Rd, np.float32(0.5))
    rng = np.random.default_rng(4)
    n, m = 97, 5
    cd = rng.integers(-5, Ed + Id + Rd + 1000, n * m).astype(np.int32)
    path = str(tmp_path / "s.csv")
    with open(path, "w") as f:
        f.write("time,simulation_id,exposed,infectious,resistant,susceptible\n")
    assert L.ref_write_state(path.encode(), None, cd, n, m, 123) == 0
    rows = np.loadtxt(path, delimiter=",", skiprows=1, dtype=np.int64).reshape(m, 6)
    for r in range(m):
        cls = [oracle.lib().orc_countdown_class(int(c), Ed, Id, Rd) for c in cd[r * n:(r + 1) * n]]
        # oracle classes: 0 S, 1 E, 2 I, 3 R; CSV columns: E, I, R, S
        want = [cls.count(1), cls.count(2), cls.count(3), cls.count(0)]
        assert list(rows[r, 2:]) == want
