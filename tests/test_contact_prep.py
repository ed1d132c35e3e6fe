"""rp_graph_from_arrays's host preparation (replay_b200/csrc/contact_prep.h):
the multithreaded version gives the sequential pass's results -- ordered
endpoints, the count of distinct nodes, and the first contact with an
endpoint out of range -- for every thread count (no GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r'''
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "contact_prep.h"

static uint64_t s = 88172645463325252ull;
static uint32_t next() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }

// the sequential pass: first bad contact, or -1 with the ordered endpoints
// and the distinct-node count
static int64_t reference(const std::vector<int32_t> &u, const std::vector<int32_t> &v, int32_t n_nodes,
                         std::vector<int32_t> &uu, std::vector<int32_t> &vv, int32_t &n_index) {
  std::vector<uint8_t> seen(n_nodes, 0);
  n_index = 0;
  for (size_t k = 0; k < u.size(); ++k) {
    if (u[k] < 0 || v[k] < 0 || u[k] >= n_nodes || v[k] >= n_nodes) return (int64_t)k;
    uu[k] = u[k] < v[k] ? u[k] : v[k];
    vv[k] = u[k] < v[k] ? v[k] : u[k];
    n_index += !seen[u[k]]; seen[u[k]] = 1;
    n_index += !seen[v[k]]; seen[v[k]] = 1;
  }
  return -1;
}

static int check(int64_t n, int32_t n_nodes, int64_t bad_at, int32_t bad_value) {
  std::vector<int32_t> u(n), v(n);
  for (int64_t k = 0; k < n; ++k) {
    u[k] = (int32_t)(next() % (uint32_t)n_nodes);
    v[k] = (int32_t)(next() % (uint32_t)n_nodes);
  }
  if (bad_at >= 0) (bad_at % 2 ? v : u)[bad_at] = bad_value;
  std::vector<int32_t> ru(n), rv(n);
  int32_t rn = -7;
  const int64_t rb = reference(u, v, n_nodes, ru, rv, rn);
  for (int threads : {1, 2, 3, 8, 16}) {
    std::vector<int32_t> pu(n), pv(n);
    int32_t pn = -7;
    const int64_t pb = rp::prep_contacts(u.data(), v.data(), n, n_nodes, pu.data(), pv.data(), &pn, threads);
    if (pb != rb) { printf("bad index %lld vs %lld (n %lld, threads %d)\n", (long long)pb, (long long)rb, (long long)n, threads); return 1; }
    if (rb < 0 && (pn != rn || pu != ru || pv != rv)) { printf("results differ (n %lld, threads %d)\n", (long long)n, threads); return 1; }
  }
  return 0;
}

int main() {
  int fails = 0;
  fails += check(0, 10, -1, 0);
  fails += check(1, 1, -1, 0);
  fails += check(1000, 50, -1, 0);
  fails += check(5000000, 100000, -1, 0);     // several ranges of 2^20 contacts
  fails += check(5000000, 3000000, -1, 0);    // nodes that never appear
  fails += check(5000000, 100000, 0, -1);     // first contact, first range
  fails += check(5000000, 100000, 1234567, 100000);   // inside the second range
  fails += check(5000000, 100000, 4999999, -5);       // last contact
  fails += check(3000000, 1000, 2999998, 1000);
  printf(fails ? "FAIL\n" : "OK\n");
  return fails != 0;
}
'''


def test_parallel_prep_matches_sequential_pass(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "prep.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "prep"
    subprocess.run([cxx, "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "replay_b200", "csrc"),
                    str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout + r.stderr
