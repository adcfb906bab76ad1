"""The host thread pool that fills and empties the pinned staging ring of
host-pointer calls (prandtl_api.cu, class CopyPool), compiled on its own with
g++ from the library source and checked on the CPU: copies of several sizes
and thread counts land exactly in place, and concurrent callers (one copy at
a time) all get their own data."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <unistd.h>
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>
%s
int main() {
    std::vector<char> a(50 << 20), b(50 << 20);
    for (size_t k = 0; k < a.size(); ++k) a[k] = (char)(k * 7 + 3);
    for (int parts : {1, 2, 8, 12, 40}) {
        for (size_t n : {size_t(100), size_t(1) << 20, (size_t(1) << 20) + 13, size_t(33) << 20}) {
            std::fill(b.begin(), b.end(), 0);
            CopyPool::get().copy(b.data() + 5, a.data() + 3, n, parts);
            if (memcmp(b.data() + 5, a.data() + 3, n) != 0 || b[4] != 0 || b[5 + n] != 0) {
                printf("FAIL parts %%d n %%zu\n", parts, n);
                return 1;
            }
        }
    }
    std::vector<std::thread> th;
    bool ok = true;
    for (int t = 0; t < 4; ++t)
        th.emplace_back([&, t] {
            std::vector<char> d(8 << 20);
            for (int r = 0; r < 20; ++r) {
                CopyPool::get().copy(d.data(), a.data() + t, d.size(), 8);
                if (memcmp(d.data(), a.data() + t, d.size())) ok = false;
            }
        });
    for (auto &x : th) x.join();
    printf(ok ? "pool ok\n" : "FAIL concurrent\n");
    return ok ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_copy_pool_copies_exactly(tmp_path):
    src = open(os.path.join(ROOT, "prandtl_b200", "csrc", "prandtl_api.cu")).read()
    m = re.search(r"class CopyPool \{.*?\n\};\n", src, re.S)
    assert m, "CopyPool not found"
    cpp = tmp_path / "pool.cpp"
    cpp.write_text(HARNESS % m.group(0))
    exe = tmp_path / "pool"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", str(cpp), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "pool ok" in r.stdout, r.stdout + r.stderr
