"""Host worker pool (tan_b200/csrc/tanb_host_pool.cpp), compiled with the host
compiler and driven without a GPU: every index runs exactly once for any job
size, jobs from several threads at once do not mix, and a child forked after
the pool started runs its jobs serially instead of waiting on threads it does
not have. copy_for_device and copy_rows_for_device (the streaming copies into
staging memory) copy every byte for any size and any source / destination
alignment, and write nothing outside the destination range."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>
#include <sys/wait.h>
#include <unistd.h>
#include "tanb_host_pool.h"

static int check(int n) {
  std::vector<std::atomic<int>> hits(n > 0 ? n : 1);
  for (auto& h : hits) h.store(0);
  tanb::host_parallel_for(n, [&](int i) { hits[i].fetch_add(1); });
  for (int i = 0; i < n; ++i)
    if (hits[i].load() != 1) return 1;
  return 0;
}

static int check_copy() {
  std::vector<unsigned char> src(70000), dst(70000 + 64);
  for (size_t i = 0; i < src.size(); ++i) src[i] = (unsigned char)(i * 131u + 7u);
  for (size_t n : {0u, 1u, 15u, 255u, 256u, 300u, 4095u, 4096u, 4097u, 4160u, 65536u + 13u})
    for (int so = 0; so < 3; ++so)
      for (int doff = 0; doff < 19; doff += 3) {
        std::fill(dst.begin(), dst.end(), (unsigned char)0xA5);
        if (so == 1) {
          tanb::copy_rows_for_device(dst.data() + 16 + doff, src.data() + so, n);
          tanb::copy_for_device_fence();
        } else {
          tanb::copy_for_device(dst.data() + 16 + doff, src.data() + so, n);
        }
        for (size_t i = 0; i < dst.size(); ++i) {
          const bool in = i >= (size_t)(16 + doff) && i < 16 + doff + n;
          const unsigned char want = in ? src[so + i - 16 - doff] : (unsigned char)0xA5;
          if (dst[i] != want) return 1;
        }
      }
  return 0;
}

int main() {
  int bad = 0;
  bad += 1000 * check_copy();
  for (int n : {0, 1, 2, 3, 7, 64, 1000, 4097}) bad += check(n);
  std::vector<std::thread> ts;
  std::atomic<int> tbad{0};
  for (int t = 0; t < 4; ++t)
    ts.emplace_back([&] { for (int r = 0; r < 50; ++r) tbad += check(37 + r); });
  for (auto& t : ts) t.join();
  bad += tbad.load();
  pid_t pid = fork();
  if (pid == 0) _exit(check(500) == 0 ? 0 : 3);
  int st = 0;
  waitpid(pid, &st, 0);
  if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad += 100;
  std::printf("bad=%d threads=%d\n", bad, tanb::host_pool_threads());
  return bad ? 1 : 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_host_pool(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    csrc = os.path.join(ROOT, "tan_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", csrc, str(src),
                    os.path.join(csrc, "tanb_host_pool.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bad=0" in r.stdout
