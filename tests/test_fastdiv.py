"""The batched multi-level kernel splits a cell index into box coordinates with FastDiv
(aa_kernel.cuh: division of 31-bit integers by an invariant divisor through a multiply and a
shift).  Its host build is checked here against exact division for every divisor up to 4096, the
box extents of the benchmark grids, and dividends at both ends of the 31-bit range."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstdint>
#include "aa_kernel.cuh"
int main() {
    unsigned long long bad = 0, checked = 0;
    const uint32_t extra[] = {4097, 65535, 65536, 65537, 257 * 129, 1u << 20, (1u << 30) + 3, 0x7fffffffu};
    auto check = [&](uint32_t d) {
        const zl::FastDiv f = zl::FastDiv::make(d);
        uint32_t seed = 12345u + d;
        for (int i = 0; i < 4000; ++i) {
            uint32_t n;
            if (i < 1000) n = (uint32_t)i;
            else if (i < 2000) n = 0x7fffffffu - (uint32_t)(i - 1000);
            else if (i < 3000) n = (uint32_t)(i - 2000) * d + (uint32_t)(i % 7) - 3u;  // around multiples
            else { seed = seed * 1664525u + 1013904223u; n = seed >> 1; }
            if (n > 0x7fffffffu) continue;
            ++checked;
            if (f.div(n) != n / d) ++bad;
        }
    };
    for (uint32_t d = 1; d <= 4096; ++d) check(d);
    for (uint32_t d : extra) check(d);
    std::printf("%llu %llu\n", checked, bad);
    return bad != 0;
}
"""


def test_fastdiv_matches_exact_division(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "fastdiv.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "fastdiv"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "zllbm_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    checked, bad = (int(v) for v in out.stdout.split())
    assert out.returncode == 0 and bad == 0 and checked > 16_000_000
