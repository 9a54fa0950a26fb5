"""CPU test of FastDiv (chll_common.cuh), the multiply-shift division the
sweep kernels use to turn a unit index into (row, plane): compiled from the
product header with the host compiler and checked against integer division
over edge cases and random pairs."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

SRC = r"""
#include <cstdio>
#include <cstdint>
#include <random>
#include "chll_common.cuh"
int main() {
  std::mt19937_64 rng(7);
  uint64_t bad = 0, n = 0;
  const uint32_t divisors[] = {1u, 2u, 3u, 5u, 7u, 8u, 12u, 16u, 24u, 60u, 120u, 128u, 240u,
                               480u, 481u, 1000u, 65535u, 65536u, 65537u, 1u << 20,
                               (1u << 20) + 1, 2147483647u, 2147483648u};
  for (uint32_t d : divisors) {
    chll::FastDiv f(d);
    const uint32_t xs[] = {0u, 1u, d - 1, d, d + 1, 2 * d - 1, 2147483646u, 2147483647u};
    for (uint32_t x : xs) { if (x < 2147483648u) { ++n; bad += f.div(x) != x / d; } }
    for (int t = 0; t < 200000; ++t) {
      const uint32_t x = (uint32_t)(rng() & 0x7fffffffu);
      ++n; bad += f.div(x) != x / d;
    }
  }
  for (int t = 0; t < 2000; ++t) {
    const uint32_t d = 1 + (uint32_t)(rng() % 0x7fffffffu);
    chll::FastDiv f(d);
    for (int u = 0; u < 200; ++u) {
      const uint32_t x = (uint32_t)(rng() & 0x7fffffffu);
      ++n; bad += f.div(x) != x / d;
    }
  }
  std::printf("%llu %llu\n", (unsigned long long)n, (unsigned long long)bad);
  return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs a host C++ compiler")
def test_fastdiv_matches_integer_division(tmp_path):
    src = tmp_path / "fastdiv.cpp"
    src.write_text(SRC)
    exe = tmp_path / "fastdiv"
    cuda_inc = "/usr/local/cuda/include"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{cuda_inc}",
                    f"-I{os.path.join(ROOT, 'chllmodel_b200', 'csrc')}", str(src), "-o", str(exe)],
                   check=True, env={**os.environ, "CC": "gcc", "CXX": "g++"})
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    n, bad = map(int, out.stdout.split())
    assert n > 1_000_000 and bad == 0
