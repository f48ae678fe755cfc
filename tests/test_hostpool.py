"""The host worker pool of the Krylov convergence checks (csrc/bd_hostpool.h).

No reference counterpart.  A C++ harness compiled from the header checks, on
the CPU, that HostPool::run calls every index exactly once and returns only
after all calls have finished: eight caller threads (replicas of a batch) each
run 3000 jobs of 1 to 24 indices against the shared workers, with calls of
uneven length; the harness runs under a time limit so that a lost wake-up
fails the test instead of hanging it.
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "smdlt-ca-chrg-flow_b200", "csrc")

HARNESS = r"""
#include "bd_hostpool.h"
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

int main() {
  std::atomic<int> bad{0};
  std::vector<std::thread> callers;
  for (int t = 0; t < 8; t++)
    callers.emplace_back([&bad, t] {
      for (int it = 0; it < 3000; it++) {
        int n = 1 + (it * 7 + t) % 24;
        std::vector<std::atomic<int>> hits(n);
        for (auto& h : hits) h.store(0);
        std::atomic<int> finished{0};
        bd::HostPool::get().run(n, [&](int i) {
          volatile double x = 0;
          for (int s = 0; s < 50 * (i % 5); s++) x = x + s;
          hits[i].fetch_add(1);
          finished.fetch_add(1);
        });
        if (finished.load() != n) bad.fetch_add(1);
        for (auto& h : hits)
          if (h.load() != 1) bad.fetch_add(1);
      }
    });
  for (auto& c : callers) c.join();
  std::printf("workers %d bad %d\n", bd::HostPool::get().workers(), bad.load());
  return bad.load() == 0 ? 0 : 1;
}
"""


def test_hostpool_runs_every_index_once(tmp_path):
    src = tmp_path / "pool.cc"
    exe = tmp_path / "pool"
    src.write_text(HARNESS)
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, str(src), "-o", str(exe)],
                   check=True)
    try:
        r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    except subprocess.TimeoutExpired:
        pytest.fail("HostPool::run did not return (lost wake-up)")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bad 0" in r.stdout
