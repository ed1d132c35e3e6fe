"""Benchmark: node-replica-steps/s of the Monte Carlo SEIR replay on B200.

One bench step = one full replay of the replica-sweep workload (N=100,000
nodes in 100 communities, 20M contacts over 14 days, 336 one-hour steps,
4,096 replicas = 64 beta values x 64 seeds, 20 initial infected) through the
batched bit-packed path with the window CSR built inside the step loop.
Extra keys report the same replay with prebuilt window CSRs and through the
plain per-replica SpMV path, the dominant kernel's HBM roofline, and the
C oracle's CPU throughput on a bounded sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With torchrun (N > 1) rank r replays replicas [r M, (r+1) M) of one job
(replica_offset): replicas shard with no data-path collective ("scaling":
"weak").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-replica-steps/s"
UNIT = "node-replica-steps/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["sweep", "small", "hot", "quiet", "dense", "uneven"],
                    default="sweep",
                    help="sweep: the replica-sweep replay (default); small: N=1,000 / 1,000 replicas; "
                         "hot: the sweep network with 5,000 initial infected for 12 steps; quiet: its "
                         "first 6 steps; dense: 3 days of the dense stress network; uneven: 32 "
                         "networks of the uneven batch for 96 steps (profiler cases)")
    ap.add_argument("--no-extras", action="store_true", help="skip plain-path / CPU / e2e legs")
    ap.add_argument("--record-traffic", metavar="NCU_CSV",
                    help="store the step kernels' DRAM bytes per step of --workload from an ncu CSV in "
                         "profiles/traffic.json and exit")
    ap.add_argument("--capture", default="", help="the ncu command line that made --record-traffic's CSV")
    return ap.parse_args()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload(name):
    from replay_b200 import synthetic
    if name == "small":
        return synthetic.small_seir()
    if name == "uneven":
        # the uneven batch's network mix (N log-uniform in 500..50,000, 128
        # replicas each) on 32 networks for 96 steps, batched into one replay
        from replay_b200 import batch_networks
        b = synthetic.uneven_batch(n_networks=32)
        s, e, u, v, n, off = batch_networks(b["networks"])
        return dict(start=s, end=e, u=u, v=v, n_nodes=n, net_first=off,
                    params=dict(b["params"], iterations=96),
                    name="uneven batch sample: 32 networks, N log-uniform 500..50k, 96 x 30 min, M=128 each")
    if name == "dense":
        # the dense stress network's per-window shape (N = 5,000, hub rows of
        # thousands of pairs, 16,384 replicas) on 3 days of its contacts, with
        # 5% initially infected so that the hub rows carry infectious replicas
        net = synthetic.dense_stress(n_contacts=5_000_000, days=3)
        net["params"] = dict(net["params"], initial_count=250, iterations=48)
        net["name"] = ("dense stress network, 3 days (5M contacts), N=5000, M=16384, "
                       "250 initial infected, 48 x 15 min")
        return net
    net = synthetic.replica_sweep()
    if name == "quiet":
        # the sweep's opening steps, where almost every replica is susceptible
        net["params"] = dict(net["params"], iterations=6)
        net["name"] += " (first 6 steps)"
    if name == "hot":
        # every step as busy as the sweep's peak: a short replay for profiler captures
        net["params"] = dict(net["params"], initial_count=5000, iterations=12)
        net["name"] += " (5,000 initial infected, 12 steps)"
    return net


TRAFFIC_JSON = os.path.join(ROOT, "profiles", "traffic.json")


def profiled_traffic(name):
    """DRAM bytes per step (k_infect + k_flow) of this workload, from profiles/traffic.json
    (written by `bench.py --record-traffic` from an ncu capture), or None."""
    try:
        with open(TRAFFIC_JSON) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return None, None
    w = d.get("workloads", {}).get(name)
    if not w:
        return None, None
    return float(w["bytes_per_launch"]), w.get("capture")


def record_traffic(csv_path, workload_name, capture):
    """Reads an ncu CSV (`ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum
    ... --csv`) and stores the DRAM bytes per step (k_infect + k_flow, one
    launch each, averaged over the first replay's steps) of the workload in
    profiles/traffic.json."""
    import csv
    with open(csv_path) as f:
        lines = [ln for ln in f if ln.startswith('"')]
    per_launch = {}
    for r in csv.DictReader(lines):
        kname = r.get("Kernel Name", "")
        if "k_infect" not in kname and "k_flow" not in kname:
            continue
        name, unit = r["Metric Name"], r.get("Metric Unit", "")
        val = float(r["Metric Value"].replace(",", ""))
        scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}.get(unit, 1)
        if name in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            k = "k_infect" if "k_infect" in kname else "k_flow"
            per_launch.setdefault(k, {})[r["ID"]] = per_launch.get(k, {}).get(r["ID"], 0.0) + val * scale
    if not per_launch.get("k_infect") or not per_launch.get("k_flow"):
        raise SystemExit(f"no k_infect / k_flow DRAM metrics in {csv_path}")
    steps = int(workload(workload_name)["params"]["iterations"])
    order = lambda d: [d[k] for k in sorted(d, key=int)][:steps]  # launch order, one replay
    inf, flo = order(per_launch["k_infect"]), order(per_launch["k_flow"])
    if len(inf) < steps or len(flo) < steps:
        raise SystemExit(f"{csv_path} holds {len(inf)} / {len(flo)} step launches, not {steps}")
    rows = [a + b for a, b in zip(inf, flo)]
    try:
        with open(TRAFFIC_JSON) as f:
            d = json.load(f)
    except (OSError, ValueError):
        d = {"kernel": "k_infect + k_flow",
             "metric": "dram__bytes_read.sum + dram__bytes_write.sum of the two launches of a step",
             "workloads": {}}
    d["workloads"][workload_name] = {"bytes_per_launch": sum(rows) / len(rows), "steps": len(rows),
                                     "k_infect": sum(inf) / len(inf), "k_flow": sum(flo) / len(flo),
                                     "min": min(rows), "max": max(rows), "capture": capture}
    with open(TRAFFIC_JSON, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
        f.write("\n")
    print(json.dumps(d["workloads"][workload_name]))


def algorithmic_bytes(n, m, steps, nnz_total):
    """Lower-bound HBM bytes of the batched step kernel over one replay:
    per step 4(N+1) CSR row pointers + 8 n_z CSR pairs + 4 W n_z gathered
    mask words + 4 W N mask writes + 2 (2/8) N M state planes read+written +
    16 M count bytes, W = ceil(M/32)."""
    w = (m + 31) // 32
    return steps * (4 * (n + 1) + 4 * w * n + 0.5 * n * m + 16 * m) + (8 + 4 * w) * nnz_total


def plain_bytes(n, m, steps, nnz_total):
    """Per-replica SpMV path, same metric: each replica re-reads the CSR and
    gathers 4 B per entry, writes 4 B exposure per node, plus state r/w."""
    return m * (steps * (4 * (n + 1) + 4 * n) + 12 * nnz_total) + steps * 0.5 * n * m


def run_ours(args, rank, world, local_rank):
    import torch

    import replay_b200

    torch.cuda.set_device(local_rank)
    dev = local_rank
    net = workload(args.workload)
    p = dict(net["params"])
    # rank r replays replicas [r M, (r + 1) M) of one N M-replica job
    p["replica_offset"] = rank * p["M"]
    n_nodes = net["n_nodes"]
    M, T = p["M"], p["iterations"]
    nrs_per_replay = n_nodes * M * T

    t0 = time.perf_counter()
    g = replay_b200.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], n_nodes, device=dev)
    ingest_s = time.perf_counter() - t0
    nets = {"networks": net["net_first"]} if "net_first" in net else {}
    sim = replay_b200.Simulation(g, path="batched", csr="per-step", **nets, **p)
    info = sim.info

    stream = torch.cuda.Stream(device=dev)

    def timed(s, k, w):
        with torch.cuda.stream(stream):
            for _ in range(w):
                s.enqueue(stream.cuda_stream)
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(k):
                s.enqueue(stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=f"cuda:{dev}")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    with ClockSampler(dev) as clk:
        ms_total = timed(sim, args.steps, args.warmup)
    clocks = clk.summary()
    ms_step = ms_total / args.steps
    value = nrs_per_replay * world / (ms_step / 1e3)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32 replica bit planes, int32/int64 exact contact-second sums",
           "data": "synthetic (seeded generator with the workload's shapes and distributions)",
           "config": {"workload": net["name"], "nodes": n_nodes, "contacts": int(len(net["start"])),
                      "replicas": M, "steps": T, "path": "batched bit-packed SpMM, window CSR built per step",
                      "parallelism": f"replicas x{world} (independent ranks)",
                      "l2": "state planes + CSRs exceed L2 (126 MB); no flush"},
           "clocks": clocks,
           "gpu_launches": info["kernels_per_run"] * args.steps}

    # ---- prebuilt-CSR variant (with --no-extras only built, for its nnz count,
    # after the per-step replays, so that those are the process's first launches) ----
    prof_ps = sim.profile() if args.no_extras else None
    sim_pre = replay_b200.Simulation(g, path="batched", csr="prebuilt", **nets, **p)
    nnz_total = sim_pre.info["nnz_total"]
    if not args.no_extras:
        ms_pre = timed(sim_pre, args.steps, 1) / args.steps
        out["prebuilt_csr"] = {"value": nrs_per_replay * world / (ms_pre / 1e3), "ms_per_step": ms_pre,
                               "prebuilt_nnz": sim_pre.info["prebuilt_nnz"]}

    # ---- roofline of the step: k_infect + k_flow, one launch each per step ----
    hbm, peak_kind = load_peaks()
    prof = prof_ps if args.no_extras else sim_pre.profile()
    bytes_replay = algorithmic_bytes(n_nodes, M, T, nnz_total)
    infect_ms = prof["spmv_ms"] / max(1, prof["spmv_launches"])
    flow_ms = prof["step_ms"] / max(1, prof["step_launches"])
    step_launch_ms = infect_ms + flow_ms
    achieved = (bytes_replay / T) / (step_launch_ms / 1e3) / 1e9
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                       "frac": achieved / hbm, "peak_source": f"{peak_kind} (copy bandwidth)",
                       "kernel": "k_infect + k_flow (the two launches of one step)",
                       "algorithmic_bytes_per_launch": bytes_replay / T,
                       "avg_launch_us": step_launch_ms * 1e3,
                       "avg_launch_us_by_kernel": {"k_infect": infect_ms * 1e3, "k_flow": flow_ms * 1e3},
                       "traffic": None}
    traffic, capture = profiled_traffic(args.workload)
    if traffic is not None:
        out["roofline"]["traffic"] = traffic
        out["roofline"]["traffic_source"] = f"profiles/traffic.json: {capture}"
    out["profile_ms"] = {"per_step": prof} if args.no_extras else {"prebuilt": prof, "per_step": sim.profile()}

    # the legs below are single-GPU measurements: a multi-GPU run (all GPUs
    # held meanwhile) reports the step line only, and no rank waits in a
    # collective the others do not enter
    if not args.no_extras and world == 1:
        # ---- plain per-replica SpMV path (drop-in), same workload ----
        sim_plain = replay_b200.Simulation(g, path="plain", csr="prebuilt", **p)
        ms_plain = timed(sim_plain, 1, 1)
        plain_value = nrs_per_replay / (ms_plain / 1e3)
        out["plain_path"] = {"value": plain_value, "ms_per_step": ms_plain,
                             "batched_over_plain": (nrs_per_replay / (ms_pre / 1e3)) / plain_value,
                             "algorithmic_bytes": plain_bytes(n_nodes, M, T, nnz_total)}
        del sim_plain
        # ---- end to end through the public API with host buffers ----
        e2e_warmup, e2e_steps = 1, 3
        h2d = sum(int(net[k].nbytes) for k in ("start", "end", "u", "v")) + 4 * M
        d2h = (T + 1) * M * 4 * 4

        # the step's inputs sit in pinned host memory, as a caller that
        # streams contact batches would keep them (staged once, untimed)
        host_in, pinned = pinned_inputs(net)

        phases = {}

        def lap(name, t0):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            phases[name] = phases.get(name, 0.0) + (t1 - t0) * 1e3
            return t1

        def e2e_once():
            t = time.perf_counter()
            ge = replay_b200.Graph.from_arrays(host_in["start"], host_in["end"], host_in["u"], host_in["v"],
                                               n_nodes, device=dev)
            t = lap("graph_ms", t)
            se = replay_b200.Simulation(ge, path="batched", csr="per-step", **p)
            t = lap("simulation_ms", t)
            c = se.run()
            t = lap("run_ms", t)
            gi, si = ge.info, se.info
            for k in ("prep_ms", "build_ms"):
                phases["graph." + k] = phases.get("graph." + k, 0.0) + gi[k]
            for k in ("setup_ms", "alloc_ms", "prebuild_ms", "capture_ms"):
                phases["simulation." + k] = phases.get("simulation." + k, 0.0) + si[k]
            se.close()
            t = lap("close_simulation_ms", t)
            ge.close()
            lap("close_graph_ms", t)
            return c

        for _ in range(e2e_warmup):
            e2e_once()
        phases.clear()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            counts = e2e_once()
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        out["e2e"] = {"value": nrs_per_replay / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                      "d2h_bytes_per_step": d2h, "s_per_step": e2e_s,
                      "includes": "contact upload + interval index build + plan + replay + counts readback",
                      "phases_ms": {k: v / e2e_steps for k, v in sorted(phases.items())},
                      "pinned_inputs": pinned, "warmup": e2e_warmup, "steps": e2e_steps}
        out["ingest_s"] = ingest_s
        assert counts.shape == (T + 1, M, 4)
        # ---- CPU baseline: the C oracle on a bounded sample ----
        out["cpu_baseline"] = cpu_baseline(net, p)
        # ---- the reference's own benchmark scenario, both executables ----
        out["reference_scenario"] = reference_scenario_leg(replay_b200)
        # ---- node-state CSV text formatted on the device ----
        out["node_state_text"] = node_text_leg(replay_b200, dev)
        # ---- uneven batch of independent networks, default and tuned tiles ----
        out["uneven_batch"] = uneven_batch_leg(replay_b200, dev, timed)
        # ---- expected-value replay: forward, adjoint, beta calibration ----
        out["meanfield"] = meanfield_leg(replay_b200, g, net, p, nnz_total, hbm)
        # ---- the reference arm's sample and rule, on our batched countdown path ----
        out["reference_sample_countdown"] = reference_sample_leg(replay_b200, dev, timed, args)
        # ---- dense stress: hub rows, 16,384 replicas ----
        del sim_pre
        out["dense_stress"] = dense_stress_leg(replay_b200, dev, timed, hbm)
    return out


def reference_sample_leg(replay_b200, dev, timed, args):
    """The reference arm's bounded sample (`bench.py --impl reference`: the
    first 5,000 nodes' contacts, 64 replicas, all 336 steps, countdown rule
    with durations equal to the geometric means) on our batched countdown
    path: the same workload and rule as the reference's CPU number."""
    net, sample, m = reference_sample(args.workload)
    p = net["params"]
    kw = reference_countdown_params(p, sample, m)
    g = replay_b200.Graph.from_arrays(sample["start"], sample["end"], sample["u"], sample["v"],
                                      sample["n_nodes"], device=dev)
    sim = replay_b200.Simulation(g, path="batched", **kw)
    ms = timed(sim, 3, 2) / 3
    out = {"workload": f"reference arm's sample: {sample['n_nodes']} nodes, {len(sample['start'])} contacts, "
                       f"{m} replicas, {p['iterations']} steps, countdown",
           "ms_per_replay": ms, "value": sample["n_nodes"] * m * p["iterations"] / (ms / 1e3), "unit": UNIT,
           "path": "batched countdown (replica codes)"}
    sim.close()
    g.close()
    return out


def dense_stress_leg(replay_b200, dev, timed, hbm):
    """The dense stress configuration at full size (N = 5,000, 50M power-law
    contacts, 2,880 x 15 min steps, 16,384 replicas, SIR): hub rows with
    thousands of CSR entries per window.  One replay after a warm-up, window
    CSRs built per step, with its own roofline over the step kernel."""
    from replay_b200 import synthetic
    net = synthetic.dense_stress()
    p = dict(net["params"])
    n, M, T = net["n_nodes"], p["M"], p["iterations"]
    t0 = time.perf_counter()
    g = replay_b200.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], n, device=dev)
    ingest = time.perf_counter() - t0
    sim = replay_b200.Simulation(g, path="batched", csr="per-step", **p)
    ms = timed(sim, 1, 1)
    prof = sim.profile()
    sim.close()
    pre = replay_b200.Simulation(g, path="batched", csr="prebuilt", **p)
    nnz_total = pre.info["nnz_total"]
    pre.close()
    bytes_replay = algorithmic_bytes(n, M, T, nnz_total)
    launch_ms = prof["spmv_ms"] / max(1, prof["spmv_launches"]) + prof["step_ms"] / max(1, prof["step_launches"])
    achieved = (bytes_replay / T) / (launch_ms / 1e3) / 1e9
    # DRAM bytes per step of the same kernels on 3 days of this network (the
    # `dense` workload: same N, M and window shape, hence the same per-step
    # state and CSR sizes)
    traffic, capture = profiled_traffic("dense")
    g.close()
    return {"workload": net["name"], "contacts": int(len(net["start"])), "ingest_s": ingest,
            "ms_per_replay": ms, "value": n * M * T / (ms / 1e3), "unit": UNIT,
            "nnz_per_step": nnz_total / T,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "kernel": "k_infect + k_flow", "algorithmic_bytes_per_launch": bytes_replay / T,
                         "avg_launch_us": launch_ms * 1e3, "traffic": traffic,
                         "traffic_source": f"profiles/traffic.json: {capture}" if capture else None,
                         "note": "the 10 MB infectious mask stays in L2: algorithmic gather bytes exceed DRAM traffic"}}


def pinned_inputs(net):
    """Copies of the contact arrays in page-locked host memory (numpy views
    of pinned torch tensors), or the arrays themselves if pinning fails;
    returns (arrays, pinned)."""
    import torch
    try:
        out = {}
        for k in ("start", "end", "u", "v"):
            a = np.ascontiguousarray(net[k])
            t = torch.empty(a.shape, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True)
            view = t.numpy()
            view[...] = a
            out[k] = view  # the view keeps the pinned tensor alive
        return out, True
    except (RuntimeError, TypeError):
        return {k: net[k] for k in ("start", "end", "u", "v")}, False


def reference_scenario_leg(replay_b200, reps=3):
    """The reference's benchmark scenario "villages", population 1,000,
    trial 1 (benchmark/benchmark_with_trials.py: 100 one-hour steps, group
    multiplier 0.1, prob_inner 0.9, prob_inter 0.05, 10,000 replicas,
    initial infected 0.5, infect prob 1.0, E = I = 3600 s, R = 0), its
    contact file regenerated byte-identically by contact_network; the whole
    `replay` process is timed end to end (parse, index, 100 steps, no CSV
    output), as the reference's benchmark times it, for this build and for
    the reference's GPU path built from its sources, on this GPU."""
    import hashlib
    from oracle import ref
    gen = os.path.join(os.path.dirname(replay_b200.CLI_PATH), "contact_network")
    env = dict(os.environ, TZ="UTC")
    seed = int(hashlib.sha256(b"villages_1000_1").hexdigest(), 16) % (10 ** 8)
    out = {"scenario": "villages, N=1,000, trial 1, 100 x 1 h, M=10,000 (countdown)",
           "published_reference_gpu_wall_s": [5.71, 5.74], "published_hardware": "not stated"}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "villages_1000_trial1.txt")
        subprocess.run([gen, "2000-01-01T00:00:00", "100", "3600", "1000", "100", "0.9", "0.05", path, str(seed)],
                       env=env, stdout=subprocess.DEVNULL, check=True)
        with open(path) as f:
            out["contacts"] = sum(1 for _ in f) - 1
        args = ["--step-size", "3600.0", "--iterations", "100", "--M", "10000", "--initial-infected", "0.5",
                "--infect-prob", "1.0", "--exposed-duration", "3600", "--infectious-duration", "3600",
                "--resistant-duration", "0", "--start-time", "946684800", "--time-step", "3600", "-q"]

        def wall(cmd):
            times = []
            for _ in range(reps):
                t0 = time.perf_counter()
                r = subprocess.run(cmd, env=env, capture_output=True)
                times.append(time.perf_counter() - t0)
                if r.returncode:
                    return None
            return statistics.median(times)

        out["ours_wall_s"] = wall([replay_b200.CLI_PATH, path] + args)
        if os.path.exists(ref.REPLAY_REF):
            out["reference_gpu_wall_s"] = wall([ref.REPLAY_REF, path] + args)
            if out["ours_wall_s"] and out["reference_gpu_wall_s"]:
                out["speedup_same_gpu"] = out["reference_gpu_wall_s"] / out["ours_wall_s"]
    return out


def node_text_leg(replay_b200, dev):
    """--node-state-out text of the small SEIR replay (N=1,000, 50,000
    contacts, 168 steps, 1,000 replicas: 169e6 lines) formatted on the
    device and handed to a callback that only counts the bytes."""
    from replay_b200 import synthetic
    net = synthetic.small_seir()
    g = replay_b200.Graph.from_arrays(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], device=dev)
    sim = replay_b200.Simulation(g, record_node_states=True, **net["params"])
    nbytes = [0]

    def count(k, ts, data):
        nbytes[0] += len(data)
        return 0

    sim.run_text(count)  # warm-up (buffers)
    nbytes[0] = 0
    t0 = time.perf_counter()
    sim.run_text(count)
    dt = time.perf_counter() - t0
    sim.close()
    g.close()
    return {"workload": "small SEIR replay, N=1,000 x M=1,000 x 169 recorded steps", "bytes": nbytes[0],
            "seconds": dt, "GBps": nbytes[0] / dt / 1e9,
            "includes": "replay + per-step classification + device formatting + D2H into pinned buffers"}


def uneven_batch_leg(replay_b200, dev, timed):
    """256 independent networks (N log-uniform in [500, 50,000], 20 N
    contacts each, 30 days, 1,440 x 30 min steps, 128 replicas each) in one
    replay: throughput with the default tiles and after the autotuner."""
    from replay_b200 import synthetic
    batch = synthetic.uneven_batch()
    p = dict(batch["params"])
    s, e, u, v, n, off = replay_b200.batch_networks(batch["networks"])
    t0 = time.perf_counter()
    g = replay_b200.Graph.from_arrays(s, e, u, v, n, device=dev)
    ingest = time.perf_counter() - t0
    sim = replay_b200.Simulation(g, networks=off, path="batched", csr="per-step", **p)
    nrs = n * p["M"] * p["iterations"]
    ms0 = timed(sim, 2, 1) / 2
    rep = sim.autotune(probe_steps=96)
    ms1 = timed(sim, 2, 1) / 2
    out = {"workload": batch["name"], "nodes": n, "contacts": int(len(s)), "networks": len(off) - 1,
           "ingest_s": ingest, "ms_per_replay_default": ms0, "value_default": nrs / (ms0 / 1e3),
           "ms_per_replay_tuned": ms1, "value_tuned": nrs / (ms1 / 1e3), "unit": UNIT, "autotune": rep}
    sim.close()
    g.close()
    return out


def meanfield_leg(replay_b200, g, net, p, nnz_total, hbm, reps=5):
    """Mean-field replay on the same network and window CSRs: N node
    probability planes over all steps, per-node susceptibility ~ U[0.5, 1.5],
    adjoint checkpoints every 24 steps.  Times one forward and one backward
    (CUDA events, after warm-up), and calibrates beta against the Monte Carlo
    daily incidence at a hidden beta = 3e-5, checked against the Monte Carlo."""
    import torch

    from replay_b200.meanfield import MeanField, calibrate_beta, daily_incidence
    n, T = net["n_nodes"], p["iterations"]
    dev = torch.device("cuda", torch.cuda.current_device())
    mf = MeanField(g, iterations=T, step_size=p["step_size"], window=p["window"], start_time=p["start_time"],
                   checkpoint_every=24)
    sus_np = np.random.default_rng(11).uniform(0.5, 1.5, n).astype(np.float32)
    sus = torch.from_numpy(sus_np).to(dev)
    k0 = p.get("initial_count", 20)
    x0 = torch.zeros(4, n, device=dev)
    x0[2] = k0 / n
    x0[0] = 1 - k0 / n
    rates = dict(p_ei=p.get("p_ei", 1 / 48), p_ir=p.get("p_ir", 1 / 120))
    beta = torch.tensor(3e-5, device=dev, requires_grad=True)

    def fwd():
        return mf(x0, beta, susceptibility=sus, **rates)

    for _ in range(2):
        inc, _ = fwd()
        inc.sum().backward()
    torch.cuda.synchronize()
    f_ms, b_ms = [], []
    for _ in range(reps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        inc, _ = fwd()
        e1.record()
        daily_incidence(inc, 24).square().sum().backward()
        e2.record()
        torch.cuda.synchronize()
        f_ms.append(e0.elapsed_time(e1))
        b_ms.append(e1.elapsed_time(e2))
    f, b = statistics.median(f_ms), statistics.median(b_ms)
    fwd_bytes = T * (4 * (n + 1) + 32 * n) + 12 * nnz_total  # CSR + gathered p_I + 4 planes read/written
    out = {"workload": "same network and CSRs, N probability planes, s_i ~ U[0.5,1.5], checkpoints every 24",
           "forward_ms": f, "backward_ms": b, "backward_over_forward": b / f,
           "forward_GBps": fwd_bytes / (f / 1e3) / 1e9, "forward_frac_of_hbm": fwd_bytes / (f / 1e3) / 1e9 / hbm}

    # calibration: Monte Carlo target at a hidden beta, mean-field fit, Monte Carlo check
    mc = dict(p)
    mc.pop("beta_per_replica", None)

    def mc_daily(b, seed):
        sim = replay_b200.Simulation(g, path="batched", csr="prebuilt",
                                     **dict(mc, beta=b, seed=seed, susceptibility=sus_np))
        c = sim.run()
        sim.close()
        S = c[:, :, 3].astype(np.float64).mean(axis=1)
        return (S[:-1] - S[1:])[: (T // 24) * 24].reshape(-1, 24).sum(1)

    hidden, beta0 = 3e-5, 1e-5
    target = mc_daily(hidden, 101)
    t0 = time.perf_counter()
    beta_cal, losses = calibrate_beta(mf, x0, target, beta0, susceptibility=sus, iters=40, lr=0.1, **rates)
    cal_s = time.perf_counter() - t0
    mc_mse = lambda b: float(((mc_daily(b, 202) - target) ** 2).mean())  # noqa: E731
    out["calibration"] = {"beta_hidden": hidden, "beta_start": beta0, "beta_calibrated": beta_cal,
                          "iterations": len(losses), "seconds": cal_s, "mf_loss_first": losses[0],
                          "mf_loss_last": losses[-1], "mc_mse_calibrated": mc_mse(beta_cal),
                          "mc_mse_start": mc_mse(beta0)}
    mf.close()
    return out


def cpu_baseline(net, p, m_sample=32, t_sample=24):
    """The oracle (single-threaded C restatement) on the same network with a
    reduced replica count and step count; loop time = t(T) - t(0)."""
    from oracle import orc
    kw = dict(n_replicas=m_sample, step_size=p["step_size"], window=p["window"], start_time=p["start_time"],
              transition=1, seed=1, beta=float(np.median(p.get("beta_per_replica", [p.get("beta", 2e-5)]))),
              p_ei=p.get("p_ei", 0.0), p_ir=p.get("p_ir", 0.0), initial_count=p.get("initial_count", 10),
              has_exposed=int(p.get("has_exposed", True)))
    t0 = time.perf_counter()
    orc.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], n_steps=0, **kw)
    t1 = time.perf_counter()
    orc.run(net["start"], net["end"], net["u"], net["v"], net["n_nodes"], n_steps=t_sample, **kw)
    t2 = time.perf_counter()
    loop = (t2 - t1) - (t1 - t0)
    return {"value": net["n_nodes"] * m_sample * t_sample / loop, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"same network, {m_sample} replicas x {t_sample} steps; loop time = t({t_sample} steps) - t(0)"}


# ---------------------------------------------------------------------------
def reference_sample(workload_name):
    """A bounded sample of the workload for the reference CPU path: the first
    5 communities (5,000 nodes) with the contacts among them, 64 replicas,
    all 336 steps, countdown durations equal to the geometric means."""
    net = workload(workload_name)
    if workload_name == "sweep":
        keep_n = 5000
        sel = (net["u"] < keep_n) & (net["v"] < keep_n)
        sample = {k: net[k][sel] for k in ("start", "end", "u", "v")}
        sample["n_nodes"] = keep_n
        m = 64
    else:
        sample = {k: net[k] for k in ("start", "end", "u", "v")}
        sample["n_nodes"] = net["n_nodes"]
        m = 100
    return net, sample, m


def reference_countdown_params(p, sample, m):
    """The countdown rule of the reference arm's sample: infect-prob from the
    sweep's median beta per contact-hour, durations equal to the geometric
    means, resistance beyond the horizon, Bernoulli initial infection at the
    workload's initial fraction."""
    beta = float(np.median(p.get("beta_per_replica", [p.get("beta", 2e-5)])))
    return dict(M=m, iterations=p["iterations"], step_size=p["step_size"], window=p["window"],
                start_time=p["start_time"], transition="countdown",
                initial_infected=p["initial_count"] / sample["n_nodes"],
                infect_prob=float(1.0 - np.exp(-beta * 3600.0)),
                exposed_duration=int(3600 / max(p.get("p_ei", 1 / 48), 1e-9)),
                infectious_duration=int(3600 / p["p_ir"]), resistant_duration=10 ** 8)


def run_reference(args):
    from oracle import ref
    from replay_b200 import synthetic
    net, sample, m = reference_sample(args.workload)
    p = net["params"]
    T = p["iterations"]
    if not os.path.exists(ref.REPLAY_REF):
        return {"impl": "reference", "unavailable": "oracle/_ref/replay_ref was not built (reference tree absent at build time)"}
    kw = reference_countdown_params(p, sample, m)
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "contacts.txt")
        synthetic.write_contact_file(path, sample)
        base = [path, "--cpu-only", "--cpu-threads", cores, "-q", "--M", m, "--step-size", kw["step_size"],
                "--static-network-duration", kw["window"], "--start-time", kw["start_time"],
                "--initial-infected", kw["initial_infected"], "--infect-prob", kw["infect_prob"],
                "--exposed-duration", kw["exposed_duration"],
                "--infectious-duration", kw["infectious_duration"],
                "--resistant-duration", kw["resistant_duration"]]
        times = []
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            r0 = ref.run_cli(base + ["--iterations", 0])
            t1 = time.perf_counter()
            r1 = ref.run_cli(base + ["--iterations", T])
            t2 = time.perf_counter()
            if r0.returncode or r1.returncode:
                return {"impl": "reference", "unavailable": f"reference exited {r0.returncode}/{r1.returncode}"}
            if it >= args.warmup:
                times.append((t2 - t1) - (t1 - t0))
    loop = statistics.median(times)
    value = sample["n_nodes"] * m * T / loop
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": loop * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 countdowns, fp32 exposures",
            "data": "synthetic", "config": {"workload": net["name"], "sample_nodes": sample["n_nodes"],
                                            "sample_contacts": int(len(sample["start"])), "replicas": m,
                                            "steps": T},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"first {sample['n_nodes']} nodes' contacts, {m} replicas, {T} steps, "
                                       "replay --cpu-only, loop = t(iterations=T) - t(iterations=0)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse_args()
    if args.record_traffic:
        record_traffic(args.record_traffic, args.workload, args.capture)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device(f"cuda:{local_rank}"))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
