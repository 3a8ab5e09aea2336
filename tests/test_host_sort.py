"""The host-side radix sort that orders a group-by's rows by group when they
are first read (capi.cu, mgv::sort_group_rows), checked on the CPU against
std::stable_sort: a small C++ program linked with libmgv.so, compiled here
with g++ (no GPU needed; the library loads without one)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_DIR = os.path.join(REPO, "multigpu-vector_b200")

SRC = r"""
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>
#include "mgv.h"
namespace mgv { void sort_group_rows(std::vector<mgv_group_row>& v); }
int main() {
    std::mt19937 g(12345);
    const size_t sizes[] = {0, 1, 2, 63, 64, 65, 4095, 4096, 4097, 70001};
    int trial = 0;
    for (size_t n : sizes)
        for (int mode = 0; mode < 4; ++mode, ++trial) {
            std::vector<mgv_group_row> v(n);
            for (size_t i = 0; i < n; ++i) {
                const uint32_t r = g();
                v[i].group = mode == 0 ? (int32_t)r                      // full range
                           : mode == 1 ? (int32_t)(r % 4096)             // small ids: one or two passes
                           : mode == 2 ? (int32_t)(r % 200) - 100        // negative and positive
                                       : (i % 3 ? INT32_MIN : INT32_MAX);  // the extremes
                v[i].sum = (int64_t)i;
                v[i].count = 1;
            }
            std::vector<mgv_group_row> w = v;
            mgv::sort_group_rows(v);
            std::stable_sort(w.begin(), w.end(), [](const mgv_group_row& a, const mgv_group_row& b) {
                return a.group < b.group;
            });
            for (size_t i = 0; i < n; ++i)
                if (v[i].group != w[i].group || (n >= 64 && v[i].sum != w[i].sum)) {
                    std::printf("mismatch: n=%zu mode=%d at %zu\n", n, mode, i);
                    return 1;
                }
        }
    std::printf("ok %d\n", trial);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_group_row_radix_sort(tmp_path):
    lib = os.path.join(LIB_DIR, "libmgv.so")
    if not os.path.exists(lib):
        pytest.skip("libmgv.so is not built")
    src = tmp_path / "sort_check.cpp"
    exe = tmp_path / "sort_check"
    src.write_text(SRC)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe),
                    "-L", LIB_DIR, "-lmgv", f"-Wl,-rpath,{LIB_DIR}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok")
