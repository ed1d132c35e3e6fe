"""Monte Carlo output against the reference's own Monte Carlo, in distribution.

The reference draws from unseeded generators (cuRAND seeded with clock64()
and time(NULL) on the GPU path; rand() reseeded with time(NULL) every step
on the CPU path, tool/gpu_cpu_temporal_sim.cu:81, 149, 365, 468), so its
trajectories cannot be matched one to one.  Both `replay` executables run
the same countdown SIR configuration on the same contact file with 10,000
replicas each; the summary CSVs are compared per time point and compartment
(two-sample z of the means against the 95% interval) and on the final
epidemic size (two-sample Kolmogorov-Smirnov).  Runs where a GPU is present,
so that the reference's GPU path can run too; needs the reference built from its
sources (oracle/_ref/replay_ref).
"""
import os
import subprocess

import numpy as np
import pytest

from replay_b200 import synthetic

pytestmark = pytest.mark.gpu

M, T = 10000, 48
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
    ours = _run(rb.CLI_PATH, graph, str(d / "ours.csv"), ["--seed", "17"], net["t0"])
    ref_gpu = _run(ref.REPLAY_REF, graph, str(d / "ref_gpu.csv"), [], net["t0"])
    ref_cpu = _run(ref.REPLAY_REF, graph, str(d / "ref_cpu.csv"), ["--cpu-only"], net["t0"])
    return ours, ref_gpu, ref_cpu


def _report(name, z, p):
    inside = float(np.mean(np.abs(z) <= 1.96))
    print(f"{name}: {inside:.3f} of mean points inside the 95% interval, max |z| {np.max(np.abs(z)):.2f}, "
          f"KS p {p:.3g}")
    return inside


def _stratified(a, b, min_count=800):
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
    return strata, np.concatenate(zs), ps


def test_matches_reference_gpu_path_in_distribution(runs):
    """The reference's GPU path seeds each (node, replica) draw with
    curand_init(clock64() + idx + seed, 0, 0): near-consecutive seeds whose
    first outputs are not independent uniforms.  Its initial-infection
    counts come out biased and overdispersed (e.g. mean 5.52-5.80 and
    variance 6.5-6.6 where Binomial(300, 0.02) gives 6.00 and 5.88, over
    10,000 replicas), and its per-step infection draws inherit the same
    seeding.  So the dynamics are compared within strata of equal initial
    count, and our output must be at least as close to the reference GPU
    path as the reference's own CPU path is (how far the GPU path strays
    varies from run to run: 32% to 88% of its means inside the 95% interval
    of its own CPU path's have been seen).  When our output and the CPU
    path's agree in distribution (the next test), the two comparisons with
    the GPU path are exchangeable and either comes out worse about half the
    time, so the bounds leave room for that spread."""
    ours, ref_gpu, ref_cpu = runs
    assert ours[-1, :, 3].mean() < 0.5 * 300  # the epidemic takes off
    k_ours, k_ref = ours[0, :, 0], ref_gpu[0, :, 0]
    print(f"initial infected: ours mean {k_ours.mean():.3f} var {k_ours.var():.3f}; "
          f"reference GPU mean {k_ref.mean():.3f} var {k_ref.var():.3f}")
    strata, z, ps = _stratified(ours, ref_gpu)
    assert len(strata) >= 3
    inside = _report(f"ours vs reference GPU path, {len(strata)} strata", z, min(ps))
    strata_c, zc, pc = _stratified(ref_cpu, ref_gpu)
    inside_c = _report(f"reference CPU vs reference GPU path, {len(strata_c)} strata", zc, min(pc))
    assert inside >= inside_c - 0.08
    assert np.max(np.abs(z)) < max(5.0, np.max(np.abs(zc)) + 1.5)
    # the final-size test is informative only in runs where the reference's
    # GPU path clearly agrees with its own CPU path (its seeding varies with
    # time)
    if min(pc) > 0.05:
        assert min(ps) > 0.01 / len(strata)


def test_matches_reference_cpu_path_in_distribution(runs):
    ours, _, ref_cpu = runs
    z, p = _compare(ours, ref_cpu)
    inside = _report("reference CPU path", z, p)
    assert inside >= 0.9 and np.max(np.abs(z)) < 5.0 and p > 0.01
