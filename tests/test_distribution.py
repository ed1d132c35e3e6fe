"""Monte Carlo output against the reference's own Monte Carlo, in distribution.

The reference draws from unseeded generators (cuRAND seeded with clock64()
and time(NULL) on the GPU path; rand() reseeded with time(NULL) every step
on the CPU path, tool/gpu_cpu_temporal_sim.cu:81, 149, 365, 468), so its
trajectories cannot be matched one to one.  Both `replay` executables run
the same countdown SEIR configuration on the same contact file, K runs of
10,000 replicas per arm (ours with K seeds; the reference's runs differ by
their clock seeds), pooled per arm.  The summary CSVs are compared per time
point and compartment (two-sample z of the means) and on the final epidemic
size (two-sample Kolmogorov-Smirnov).

These tests are statistical: they run after every bit-exact test
(tests/conftest.py orders tests marked `montecarlo` last, before the
allocation-free entry point's test), and each bound is set so that a correct
implementation fails it well under 1% of the time.  Needs a GPU (the
reference's GPU path) and the reference built from its sources
(oracle/_ref/replay_ref).
"""
import os
import subprocess
import time

import numpy as np
import pytest

from replay_b200 import synthetic

pytestmark = [pytest.mark.gpu, pytest.mark.montecarlo]

M, T, K = 10000, 48, 3
ARGS = ["--M", M, "--iterations", T, "--step-size", 3600, "--static-network-duration", 3600,
        "--initial-infected", 0.02, "--infect-prob", 0.4, "--exposed-duration", 7200,
        "--infectious-duration", 28800, "--resistant-duration", 100000000]


def _read(path):
    rows = np.loadtxt(path, delimiter=",", skiprows=1, dtype=np.int64)
    return rows[:, 2:].reshape(T + 1, M, 4)  # exposed, infectious, resistant, susceptible


def _run(exe, graph, out, extra, t0):
    cmd = [exe, graph, "-q", "--summary-out", out, "--start-time", str(t0)] + [str(a) for a in ARGS] + extra
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return _read(out)


def _compare(a, b):
    ma, mb = a.mean(axis=1), b.mean(axis=1)
    va, vb = a.var(axis=1, ddof=1), b.var(axis=1, ddof=1)
    se = np.sqrt(va / a.shape[1] + vb / b.shape[1])
    z = np.where(se > 0, (ma - mb) / np.where(se > 0, se, 1), np.where(ma == mb, 0.0, np.inf))
    from scipy.stats import ks_2samp
    final_a = a[-1, :, 2] + a[-1, :, 1] + a[-1, :, 0]  # ever infected by the end
    final_b = b[-1, :, 2] + b[-1, :, 1] + b[-1, :, 0]
    return z, ks_2samp(final_a, final_b).pvalue


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import ref
    if not ref.available() or not os.path.exists(ref.REPLAY_REF):
        pytest.skip("reference not built (oracle/_ref/replay_ref)")
    import replay_b200 as rb
    d = tmp_path_factory.mktemp("dist")
    net = synthetic.tiny(seed=123, n_nodes=300, n_contacts=9000, span=T * 3600, max_dur=3000)
    graph = str(d / "graph.txt")
    synthetic.write_contact_file(graph, net)
    ours, ref_gpu, ref_cpu = [], [], []
    for k in range(K):
        ours.append(_run(rb.CLI_PATH, graph, str(d / f"ours{k}.csv"), ["--seed", str(17 + k)], net["t0"]))
        ref_gpu.append(_run(ref.REPLAY_REF, graph, str(d / f"ref_gpu{k}.csv"), [], net["t0"]))
        # the CPU path seeds rand() with time(NULL): runs must start in different seconds
        time.sleep(1.1)
        ref_cpu.append(_run(ref.REPLAY_REF, graph, str(d / f"ref_cpu{k}.csv"), ["--cpu-only"], net["t0"]))
    return ours, ref_gpu, ref_cpu


def _report(name, z, p):
    inside = float(np.mean(np.abs(z) <= 1.96))
    rms = float(np.sqrt(np.mean(z ** 2)))
    print(f"{name}: {inside:.3f} of mean points inside the 95% interval, rms z {rms:.2f}, "
          f"max |z| {np.max(np.abs(z)):.2f}, KS p {p:.3g}")
    return inside, rms


def _stratified(a, b, min_count=1500):
    """Per-(t, compartment) z of the means and final-size KS p-values within
    strata of equal initial-infection count (initial infected show as exposed
    at t0)."""
    ka, kb = a[0, :, 0], b[0, :, 0]
    strata = [k for k in np.intersect1d(ka, kb) if (ka == k).sum() >= min_count and (kb == k).sum() >= min_count]
    zs, ps = [], []
    for k in strata:
        z, p = _compare(a[:, ka == k], b[:, kb == k])
        zs.append(z[1:])  # t0 is the stratum itself
        ps.append(p)
    return strata, (np.concatenate(zs) if zs else np.zeros(0)), ps


def test_matches_reference_cpu_path_in_distribution(runs):
    """Pooled runs of ours against pooled runs of the reference's CPU path.
    Under agreement every z is standard normal; the bounds are Bonferroni
    over the 196 (time, compartment) points (max |z| < 4.5: about 0.1% false
    failures) and a KS level of 1e-3."""
    ours, _, ref_cpu = runs
    a, b = np.concatenate(ours, axis=1), np.concatenate(ref_cpu, axis=1)
    assert a[-1, :, 3].mean() < 0.5 * 300  # the epidemic takes off
    z, p = _compare(a, b)
    _report(f"ours vs reference CPU path, {K} x {M} replicas each", z, p)
    for k in range(K):
        _report(f"  run {k}", *_compare(ours[k], ref_cpu[k]))
    assert np.max(np.abs(z)) < 4.5 and p > 1e-3


def test_matches_reference_gpu_path_in_distribution(runs):
    """The reference's GPU path seeds each (node, replica) draw with
    curand_init(clock64() + idx + seed, 0, 0): near-consecutive seeds whose
    first outputs are not independent uniforms.  Its initial-infection
    counts come out biased and overdispersed, and its per-step infection
    draws inherit the same seeding, by an amount that changes from run to
    run.  So the dynamics are compared within strata of equal initial count,
    against K pooled GPU runs, and our output must be about as close to the
    reference GPU path as the reference's own CPU path is.

    When ours and the CPU path agree in distribution (the test above), the
    two comparisons with the GPU path are exchangeable: with the GPU path's
    bias b (in standard errors) the rms z of either is about sqrt(b^2 + 1)
    and they differ by a standard normal at most (fully correlated points).
    The bounds (1.25 x the CPU path's rms z + 2.5, and 1.25 x its max |z| +
    3) leave that room, so a correct implementation fails them in well
    under 1% of runs; a rule error moves our z by tens of standard errors."""
    ours, ref_gpu, ref_cpu = runs
    a = np.concatenate(ours, axis=1)
    g = np.concatenate(ref_gpu, axis=1)
    c = np.concatenate(ref_cpu, axis=1)
    k_ours, k_ref = a[0, :, 0], g[0, :, 0]
    print(f"initial infected: ours mean {k_ours.mean():.3f} var {k_ours.var():.3f}; "
          f"reference GPU mean {k_ref.mean():.3f} var {k_ref.var():.3f}")
    strata, z, ps = _stratified(a, g)
    assert len(strata) >= 3
    inside, rms = _report(f"ours vs reference GPU path, {len(strata)} strata", z, min(ps))
    strata_c, zc, pc = _stratified(c, g)
    inside_c, rms_c = _report(f"reference CPU vs reference GPU path, {len(strata_c)} strata", zc, min(pc))
    # each GPU run on its own (diagnostics only: a run holds a third of the
    # pooled replicas, so its strata are smaller)
    for k in range(K):
        for name, x in (("ours", a), ("reference CPU", c)):
            zk = _stratified(x, ref_gpu[k], min_count=1500 // K)[1]
            if zk.size:
                _report(f"  GPU run {k}: {name}", zk, 1.0)
    assert rms < 1.25 * rms_c + 2.5
    assert np.max(np.abs(z)) < 1.25 * np.max(np.abs(zc)) + 3.0
