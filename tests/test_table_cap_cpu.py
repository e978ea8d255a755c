"""The hash-table capacity of csrc/lv_device.cuh (`table_cap`, written in closed form from the
leading zeros of k - 1) equals its definition -- twice the smallest power of two that holds
min(d, n_graph) keys, at least 2 -- over every row length up to 2^22 and sampled lengths up to
2^30 (the engine's limit on CSR entries). The kernels size every shared-memory and global
table with it, and a table smaller than twice its distinct keys would overflow. Compiled with
nvcc as host code (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "louvain-fast-move-cuda_b200", "csrc")

SRC = r"""
#include <cstdio>
#include "lv_device.cuh"

static uint32_t by_definition(uint32_t d, uint32_t ng) {
  uint32_t k = d < ng ? d : ng;
  if (k < 1) k = 1;
  uint32_t p = 2;
  while (p < 2u * k) p <<= 1;
  return p;
}

int main() {
  const uint32_t big = 1u << 30;
  for (uint32_t d = 0; d <= (1u << 22); ++d) {
    const uint32_t ng = (d * 7919u) % (1u << 22) + 1u;
    if (lv::table_cap(d, ng) != by_definition(d, ng) || lv::table_cap(d, big) != by_definition(d, big)) {
      std::printf("mismatch at d=%u\n", d);
      return 1;
    }
  }
  for (uint64_t k = 1u << 22; k <= big; k += 12347u) {
    const uint32_t d = (uint32_t)k;
    if (lv::table_cap(d, big) != by_definition(d, big) || lv::table_cap(big, d) != by_definition(big, d)) {
      std::printf("mismatch at k=%u\n", d);
      return 1;
    }
  }
  std::printf("ok\n");
  return 0;
}
"""


def test_table_cap_closed_form_equals_definition(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "table_cap.cu"
    src.write_text(SRC)
    exe = tmp_path / "table_cap"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", CSRC, str(src), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=300)
    assert out.stdout.strip() == "ok"
