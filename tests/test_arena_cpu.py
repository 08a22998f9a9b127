"""The serving loop's device-memory sub-allocator (gct_b200/csrc/arena.hpp), compiled with g++
and exercised on the CPU: first fit, alignment, coalescing, peak accounting, exhaustion."""
import shutil
import subprocess
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parents[1] / "gct_b200" / "csrc"

PROGRAM = r"""
#include "arena.hpp"
#include <cassert>
#include <cstdio>
#include <random>
#include <vector>
int main() {
    gct::Arena a(1 << 20);
    assert(a.size() == (1u << 20));
    size_t x = a.alloc(1000), y = a.alloc(1), z = a.alloc(4096);
    assert(x == 0 && y == 1024 && z == 1280);             // 256-byte granules, first fit
    assert(a.in_use() == 1024 + 256 + 4096);
    assert(a.release(y) && !a.release(y));                 // double free refused
    size_t w = a.alloc(200);
    assert(w == 1024);                                     // reuses the hole
    assert(a.release(x) && a.release(w) && a.release(z));
    assert(a.in_use() == 0 && a.free_blocks() == 1);       // fully coalesced
    assert(a.alloc((1 << 20) + 1) == SIZE_MAX);            // larger than the arena
    assert(!a.fits((1 << 20) + 1) && a.fits(1 << 20));
    // random churn: live blocks never overlap, everything coalesces back
    std::mt19937 rng(7);
    std::vector<std::pair<size_t, size_t>> live;
    for (int it = 0; it < 20000; ++it) {
        if (live.empty() || (rng() % 3)) {
            size_t n = 1 + rng() % 50000;
            size_t off = a.alloc(n);
            if (off == SIZE_MAX) continue;
            for (auto &l : live) assert(off + gct::Arena::round_up(n) <= l.first || l.first + l.second <= off);
            live.push_back({off, gct::Arena::round_up(n)});
        } else {
            size_t k = rng() % live.size();
            assert(a.release(live[k].first));
            live.erase(live.begin() + k);
        }
        assert(a.peak() >= a.in_use() && a.in_use() <= a.size());
    }
    for (auto &l : live) assert(a.release(l.first));
    assert(a.in_use() == 0 && a.free_blocks() == 1 && a.live_blocks() == 0);
    std::puts("ok");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_arena(tmp_path):
    src = tmp_path / "arena_test.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "arena_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(CSRC), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "ok"
