"""bench.py's DRAM-traffic bookkeeping (no GPU): record_traffic reads an ncu
CSV of the two step kernels, keeps the first replay's steps in launch order,
and profiled_traffic hands the per-step bytes back to the bench line."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _csv(path, launches):
    head = '"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size",' \
           '"Grid Size","Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"\n'
    with open(path, "w") as f:
        f.write("==PROF== Connected to process 1\n")
        f.write(head)
        for i, (kernel, rd, wr) in enumerate(launches):
            for name, unit, val in (("dram__bytes_read.sum", "byte", rd), ("dram__bytes_write.sum", "Mbyte", wr),
                                    ("gpu__time_duration.sum", "ns", 1000)):
                f.write(f'"{i}","1","python","h","{kernel}(PackedLayout, int)","1","7","(256, 1, 1)",'
                        f'"(443, 1, 1)","0","10.0","Command line profiler metrics","{name}","{unit}","{val:,}"\n')


def test_record_and_read_traffic(tmp_path, monkeypatch):
    bench = _bench()
    monkeypatch.setattr(bench, "TRAFFIC_JSON", str(tmp_path / "traffic.json"))
    monkeypatch.setattr(bench, "workload", lambda name: {"params": {"iterations": 2}})
    # two steps of one replay, then the first step of the next (ignored);
    # another kernel in between is skipped
    launches = [("rp::k_infect", 100, 1), ("rp::k_hits", 999, 9), ("rp::k_flow", 200, 2),
                ("rp::k_infect", 300, 3), ("rp::k_flow", 400, 4),
                ("rp::k_infect", 7777, 7), ("rp::k_flow", 8888, 8)]
    csv_path = tmp_path / "launches.csv"
    _csv(csv_path, launches)
    bench.record_traffic(str(csv_path), "sweep", "ncu ... launches.csv")
    per_step, capture = bench.profiled_traffic("sweep")
    # step 1: 100 + 1e6 + 200 + 2e6 bytes; step 2: 300 + 3e6 + 400 + 4e6
    want = ((100 + 1e6 + 200 + 2e6) + (300 + 3e6 + 400 + 4e6)) / 2
    assert abs(per_step - want) < 1e-6 and capture == "ncu ... launches.csv"
    assert bench.profiled_traffic("quiet") == (None, None)


def test_algorithmic_bytes_formula():
    bench = _bench()
    n, m, steps, nnz = 1000, 64, 3, 5000
    w = 2
    per_step = 4 * (n + 1) + 4 * w * n + 0.5 * n * m + 16 * m
    assert bench.algorithmic_bytes(n, m, steps, nnz) == steps * per_step + (8 + 4 * w) * nnz
