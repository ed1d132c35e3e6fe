"""Seeded synthetic temporal contact networks with the shapes, sizes and
value distributions of the benchmark workloads (no public dataset is used).

All generators return dict(start, end, u, v, n_nodes, ...) with int64 UTC
seconds and compressed node indices u < v (uniformly random distinct pairs
unless stated), ready for Graph.from_arrays, plus the replay parameters of
the workload under "params".
"""
import numpy as np

EPOCH_2000 = 946684800  # 2000-01-01T00:00:00Z
DAY = 86400


def _pairs_uniform(rng, n_nodes, n):
    a = rng.integers(0, n_nodes, n, dtype=np.int64)
    b = rng.integers(0, n_nodes - 1, n, dtype=np.int64)
    b = b + (b >= a)  # distinct
    return np.minimum(a, b).astype(np.int32), np.maximum(a, b).astype(np.int32)


def small_seir(seed=1, n_nodes=1000, n_contacts=50_000, days=7, steps=168, replicas=1000):
    """N=1,000 nodes, 50,000 contacts over 7 days, lognormal durations
    (median 600 s, sigma 1.0) clipped to [1 s, 8 h], 1 h steps, beta 2e-5,
    E->I / I->R geometric with means 48 h / 120 h, 10 initial infected."""
    rng = np.random.default_rng(seed)
    u, v = _pairs_uniform(rng, n_nodes, n_contacts)
    start = EPOCH_2000 + rng.integers(0, days * DAY, n_contacts, dtype=np.int64)
    dur = np.clip(np.rint(np.exp(np.log(600.0) + 1.0 * rng.standard_normal(n_contacts))), 1, 8 * 3600)
    end = start + dur.astype(np.int64)
    params = dict(M=replicas, iterations=steps, step_size=3600.0, window=3600, start_time=EPOCH_2000,
                  transition="geometric", beta=2e-5, p_ei=1 / 48, p_ir=1 / 120, initial_count=10)
    return dict(start=start, end=end, u=u, v=v, n_nodes=n_nodes, params=params,
                name="small SEIR: N=1000, 50k contacts, 168 x 1 h, M=1000")


def replica_sweep(seed=2, n_nodes=100_000, communities=100, n_contacts=20_000_000, days=14, steps=336,
                  betas=64, seeds=64):
    """N=100,000 in 100 communities of 1,000; 20M contacts, 90% within a
    community; starts over 14 days thinned by 1 + 0.8 sin(2 pi t / 24 h);
    lognormal durations (median 900 s, sigma 1.2); 1 h steps; 4,096
    replicas = 64 betas log-spaced in [5e-6, 1e-4] x 64 seeds; 20 initial
    infected per replica."""
    rng = np.random.default_rng(seed)
    size = n_nodes // communities
    intra = rng.random(n_contacts) < 0.9
    n_in = int(intra.sum())
    comm = rng.integers(0, communities, n_in, dtype=np.int64)
    a = rng.integers(0, size, n_in, dtype=np.int64)
    b = rng.integers(0, size - 1, n_in, dtype=np.int64)
    b = b + (b >= a)
    u = np.empty(n_contacts, np.int32)
    v = np.empty(n_contacts, np.int32)
    u[intra] = (comm * size + np.minimum(a, b)).astype(np.int32)
    v[intra] = (comm * size + np.maximum(a, b)).astype(np.int32)
    uu, vv = _pairs_uniform(rng, n_nodes, n_contacts - n_in)
    u[~intra], v[~intra] = uu, vv
    span = days * DAY
    # thinning: candidate times uniform, accepted with rate(t) / max rate
    starts = np.empty(0, np.int64)
    while len(starts) < n_contacts:
        need = int((n_contacts - len(starts)) * 1.9) + 1024
        t = rng.integers(0, span, need, dtype=np.int64)
        keep = rng.random(need) * 1.8 < 1.0 + 0.8 * np.sin(2 * np.pi * t / DAY)
        starts = np.concatenate([starts, t[keep]])
    start = EPOCH_2000 + np.sort(starts[:n_contacts])
    rng.shuffle(start)
    dur = np.maximum(1, np.rint(np.exp(np.log(900.0) + 1.2 * rng.standard_normal(n_contacts))))
    end = start + dur.astype(np.int64)
    beta = np.repeat(np.logspace(np.log10(5e-6), np.log10(1e-4), betas), seeds).astype(np.float32)
    params = dict(M=betas * seeds, iterations=steps, step_size=3600.0, window=3600, start_time=EPOCH_2000,
                  transition="geometric", beta_per_replica=beta, p_ei=1 / 48, p_ir=1 / 120,
                  initial_count=20)
    return dict(start=start, end=end, u=u, v=v, n_nodes=n_nodes, params=params,
                name="replica sweep: N=100k (100 communities), 20M contacts, 336 x 1 h, M=4096 (64 beta x 64 seeds)")


def dense_stress(seed=5, n_nodes=5000, n_contacts=50_000_000, days=30, steps=2880, replicas=16384):
    """N=5,000; 50M contacts with endpoints drawn by power-law activity
    (Pareto exponent 2.2, minimum 1); starts over 30 days; exponential
    durations (mean 1,200 s) clipped at 12 h; 15 min steps; 16,384 replicas;
    beta 1e-5, recovery mean 72 h, SIR; 5 initial infected."""
    rng = np.random.default_rng(seed)
    act = (rng.pareto(1.2, n_nodes) + 1.0)  # density ~ x^-2.2 for x >= 1
    p = act / act.sum()
    cdf = np.cumsum(p)
    a = np.searchsorted(cdf, rng.random(n_contacts) * cdf[-1]).astype(np.int64)
    b = np.searchsorted(cdf, rng.random(n_contacts) * cdf[-1]).astype(np.int64)
    same = a == b
    while same.any():
        b[same] = np.searchsorted(cdf, rng.random(int(same.sum())) * cdf[-1])
        same = a == b
    u, v = np.minimum(a, b).astype(np.int32), np.maximum(a, b).astype(np.int32)
    start = EPOCH_2000 + rng.integers(0, days * DAY, n_contacts, dtype=np.int64)
    dur = np.clip(np.rint(rng.exponential(1200.0, n_contacts)), 1, 12 * 3600).astype(np.int64)
    end = start + dur
    params = dict(M=replicas, iterations=steps, step_size=900.0, window=900, start_time=EPOCH_2000,
                  transition="geometric", beta=1e-5, p_ir=1 / 288, has_exposed=False, initial_count=5)
    return dict(start=start, end=end, u=u, v=v, n_nodes=n_nodes, params=params,
                name="dense stress SIR: N=5000, 50M power-law contacts, 2880 x 15 min, M=16384")


def uneven_batch(seed=3, n_networks=256, days=30, steps=1440, replicas=128):
    """256 independent networks, node counts log-uniform in [500, 50,000],
    20 x N uniform contacts each, starts over 30 days, lognormal durations
    (median 300 s, sigma 1.0), 30 min steps, 128 replicas per network,
    beta 3e-5, incubation mean 36 h, recovery mean 96 h."""
    rng = np.random.default_rng(seed)
    sizes = np.rint(np.exp(rng.uniform(np.log(500), np.log(50000), n_networks))).astype(np.int64)
    nets = []
    for n in sizes:
        m = 20 * int(n)
        u, v = _pairs_uniform(rng, int(n), m)
        start = EPOCH_2000 + rng.integers(0, days * DAY, m, dtype=np.int64)
        dur = np.maximum(1, np.rint(np.exp(np.log(300.0) + rng.standard_normal(m)))).astype(np.int64)
        nets.append(dict(start=start, end=start + dur, u=u, v=v, n_nodes=int(n)))
    params = dict(M=replicas, iterations=steps, step_size=1800.0, window=1800, start_time=EPOCH_2000,
                  transition="geometric", beta=3e-5, p_ei=1 / 72, p_ir=1 / 192, initial_count=10)
    return dict(networks=nets, params=params,
                name="uneven batch: 256 networks, N log-uniform 500..50k, 1440 x 30 min, M=128 each")


def tiny(seed=0, n_nodes=40, n_contacts=400, span=6 * 3600, max_dur=5400, negative=False):
    """Small random network for parity tests (optionally with pre-1970 times)."""
    rng = np.random.default_rng(seed)
    u, v = _pairs_uniform(rng, n_nodes, n_contacts)
    base = -span // 2 if negative else EPOCH_2000
    start = base + rng.integers(0, span, n_contacts, dtype=np.int64)
    end = start + rng.integers(1, max_dur, n_contacts, dtype=np.int64)
    return dict(start=start, end=end, u=u, v=v, n_nodes=n_nodes, t0=int(base))


def write_contact_file(path, net, ids=None):
    """Writes the NODE_LIST text format (node ids default to 0..N-1)."""
    import datetime as _dt

    n = net["n_nodes"]
    ids = np.arange(n) if ids is None else np.asarray(ids)

    def iso(t):
        return _dt.datetime.fromtimestamp(int(t), _dt.timezone.utc).strftime("%Y-%m-%dT%H:%M:%SZ")

    with open(path, "w") as f:
        f.write("NODE_LIST " + " ".join(str(int(x)) for x in ids) + "\n")
        for s, e, a, b in zip(net["start"], net["end"], net["u"], net["v"]):
            f.write(f"{int(ids[a])}, {int(ids[b])}, {iso(s)}, {iso(e)};\n")
