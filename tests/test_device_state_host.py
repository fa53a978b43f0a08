"""Per-device bookkeeping of the library's set-once state (csrc/device_state.hpp), on the CPU.

CUDA keeps a kernel's dynamic-shared-memory limit per device, so the library records each limit
it raised by (kernel, device ordinal): a limit set while device 0 was current must be set again
on device 1. The table is plain C++; this test compiles it with a fake setter and checks that
the setter runs once per (kernel, device, larger size), and that the per-device slots of
PerDevice are distinct and bounded."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "gpu-randomized-pseudoskeleton_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <thread>
#include <vector>
#include "device_state.hpp"
using namespace pskel;
static int calls = 0;
static int k1, k2;  // stand-ins for two kernels
static bool set_ok(size_t) { ++calls; return true; }
#define CHECK(c) do { if (!(c)) { std::printf("FAIL line %d\n", __LINE__); return 1; } } while (0)
int main() {
    SmemAttrTable t;
    CHECK(t.raise(&k1, 0, 100000, set_ok) && calls == 1);
    CHECK(t.raise(&k1, 0, 100000, set_ok) && calls == 1);   // same device: nothing to do
    CHECK(t.raise(&k1, 0, 50000, set_ok) && calls == 1);    // smaller need: limit kept
    CHECK(t.raise(&k1, 1, 100000, set_ok) && calls == 2);   // another device: set again
    CHECK(t.raise(&k2, 1, 100000, set_ok) && calls == 3);   // another kernel
    CHECK(t.raise(&k1, 1, 200000, set_ok) && calls == 4);   // larger need: raised
    CHECK(t.recorded(&k1, 0) == 100000 && t.recorded(&k1, 1) == 200000);
    CHECK(t.recorded(&k2, 0) == 0);
    // a failing setter records nothing
    CHECK(!t.raise(&k2, 3, 1000, [](size_t) { return false; }));
    CHECK(t.recorded(&k2, 3) == 0);
    // concurrent raises from several host threads set each (kernel, device) once
    calls = 0;
    SmemAttrTable u;
    std::vector<std::thread> th;
    for (int i = 0; i < 8; ++i)
        th.emplace_back([&u, i] { for (int d = 0; d < 4; ++d) u.raise(&k1, d, 4096, set_ok); });
    for (auto &x : th) x.join();
    CHECK(calls == 4);
    PerDevice<int> pd;
    CHECK(pd.get(0) && pd.get(1) && pd.get(0) != pd.get(1));
    CHECK(pd.get(kMaxDevices - 1) && !pd.get(kMaxDevices) && !pd.get(-1));
    std::printf("ok\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_smem_attribute_table_is_keyed_by_device(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    subprocess.run(["g++", "-std=c++17", "-O1", "-pthread", "-I", CSRC, str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
