"""The multiply-shift divisor (FDiv in csrc/cdd_internal.cuh) used for FFT and tile indexing in the
kernels: a host program built by nvcc from the same header (it makes no CUDA calls, so it runs
without a GPU) checks it against integer division on small, edge and random numerators for
divisors 1..4999 and some large ones."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "cuda-plasticity_b200", "csrc")

PROG = r'''
#include <cstdio>
#include <random>
#include "cdd_internal.cuh"
using namespace cdd;
int main() {
    std::mt19937_64 g(1);
    long long bad = 0, tot = 0;
    auto chk = [&](const FDiv& f, int n) { ++tot; if (fdiv_q(f, n) != n / f.d) ++bad; };
    for (int d = 1; d < 5000; ++d) {
        const FDiv f = fdiv_make(d);
        for (int k = 0; k < 400; ++k) chk(f, k * 7 + (int)(g() % 13));
        for (int k = 0; k < 400; ++k) chk(f, (int)(g() & 0x7fffffff));
        for (int n : {0x7fffffff, 0x7ffffffe, d - 1, d, d + 1, 2 * d - 1, 2 * d}) chk(f, n);
    }
    for (int d : {65536, 393216, 12582912, 1 << 30, 0x7fffffff}) {
        const FDiv f = fdiv_make(d);
        for (int k = 0; k < 20000; ++k) chk(f, (int)(g() & 0x7fffffff));
        chk(f, 0x7fffffff);
    }
    std::printf("%lld %lld\n", tot, bad);
    return bad != 0;
}
'''


def test_fdiv_is_exact(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc is missing")
    src = tmp_path / "fdiv.cu"
    src.write_text(PROG)
    exe = tmp_path / "fdiv"
    r = subprocess.run([nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "--expt-relaxed-constexpr", "-I", CSRC, str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    tot, bad = map(int, out.stdout.split())
    assert out.returncode == 0 and bad == 0 and tot > 4_000_000
