"""The C entry points' exception guard (tpe::guarded in tpe_internal.h) on CPU:
a C++ exception from an entry point's body becomes a status and a message,
never an exception through the C ABI. Host code only; no device call."""
from __future__ import annotations

import os
import subprocess

import pytest

from repulsive_test2_b200 import build as B

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "repulsive_test2_b200",
                    "csrc")

PROGRAM = r"""
#include <cstdio>
#include "tpe_internal.h"
namespace tpe {
void set_error(tpe_ctx* ctx, int32_t, const std::string& msg) {
    if (ctx) ctx->err = msg;
}
}  // namespace tpe
int main() {
    using namespace tpe;
    tpe_ctx* ctx = new tpe_ctx();
    int bad = 0;
    bad |= (guarded(ctx, [&]() -> int32_t { return 7; }) != 7) << 0;
    bad |= (guarded(ctx, [&]() -> int32_t { throw std::bad_alloc(); }) != TPE_ERR_OUT_OF_MEMORY) << 1;
    bad |= (ctx->err != "host allocation failed") << 2;
    bad |= (guarded(ctx, [&]() -> int32_t {
                std::vector<double> v;
                v.reserve(v.max_size() + 1);
                return 0;
            }) != TPE_ERR_TOO_LARGE) << 3;
    bad |= (guarded(ctx, [&]() -> int32_t { throw std::runtime_error("boom"); }) != TPE_ERR_INTERNAL) << 4;
    bad |= (ctx->err != "boom") << 5;
    bad |= (guarded(nullptr, [&]() -> int32_t { throw 3; }) != TPE_ERR_INTERNAL) << 6;
    printf("%d\n", bad);
    return bad != 0;
}
"""


def test_guard_turns_exceptions_into_status(tmp_path):
    src = tmp_path / "guard.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "guard"
    r = subprocess.run([B.nvcc(), *B.ARCH, "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr[-2000:])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout + out.stderr


MUTEX_PROGRAM = r"""
#include <atomic>
#include <chrono>
#include <cstdio>
#include <thread>
#include "tpe_internal.h"
namespace tpe {
void set_error(tpe_ctx* ctx, int32_t, const std::string& msg) {
    if (ctx) ctx->err = msg;
}
}  // namespace tpe
int main() {
    using namespace tpe;
    tpe_ctx* ctx = new tpe_ctx();
    std::atomic<int> inside{0}, overlaps{0}, calls{0};
    auto worker = [&]() {
        for (int i = 0; i < 200; i++) {
            guarded(ctx, [&]() -> int32_t {
                if (inside.fetch_add(1) != 0) overlaps++;
                // an entry point may call another on the same context
                guarded(ctx, [&]() -> int32_t { return 0; });
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                inside.fetch_sub(1);
                calls++;
                return 0;
            });
        }
    };
    std::thread a(worker), b(worker);
    a.join();
    b.join();
    printf("%d %d\n", overlaps.load(), calls.load());
    return overlaps.load() != 0 || calls.load() != 400;
}
"""


def test_context_calls_from_two_threads_do_not_overlap(tmp_path):
    src = tmp_path / "mutex.cu"
    src.write_text(MUTEX_PROGRAM)
    exe = tmp_path / "mutex"
    r = subprocess.run([B.nvcc(), *B.ARCH, "-std=c++17", "-I", CSRC, str(src), "-o", str(exe), "-lpthread"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr[-2000:])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "0 400", out.stdout + out.stderr
