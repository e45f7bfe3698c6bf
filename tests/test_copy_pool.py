"""The host copy threads of the irregular and regular calls (csrc/copy_pool.h),
compiled on their own with g++ and driven from a small C++ program: every
part of every job runs exactly once, arm() wakes sleeping helpers without
running anything, the pool restarts after stop(), and one part runs on the
calling thread alone."""
import os
import shutil
import subprocess
import textwrap

import pytest

CSRC = os.path.join(os.path.dirname(__file__), "..", "nbody6ppgpu-beijing_b200", "csrc")

PROGRAM = textwrap.dedent(r"""
    #include "copy_pool.h"
    #include <atomic>
    #include <cstdio>
    #include <vector>
    int main(int argc, char **argv) {
        const int want = atoi(argv[1]);
        CopyPool pool;
        for (int cycle = 0; cycle < 3; ++cycle) {
            pool.start(want);
            const int np = pool.parts();
            if (np != want) { printf("parts %d != %d\n", np, want); return 1; }
            std::vector<std::atomic<int>> hits(np);
            for (int job = 0; job < 2000; ++job) {
                if (job % 7 == 0) pool.arm();
                if (job % 500 == 0) std::this_thread::sleep_for(std::chrono::milliseconds(5));  // helpers asleep
                pool.run([&](int p) { hits[p].fetch_add(1); });
            }
            for (int p = 0; p < np; ++p)
                if (hits[p].load() != 2000) { printf("part %d ran %d times\n", p, hits[p].load()); return 1; }
            // a job's parts see the caller's data and see each other's results after run()
            std::vector<long> out(np, 0);
            pool.run([&](int p) { out[p] = 1000L * (p + 1); });
            long sum = 0;
            for (long v : out) sum += v;
            if (sum != 500L * np * (np + 1)) { printf("sum %ld\n", sum); return 1; }
            pool.stop();
        }
        printf("ok\n");
        return 0;
    }
""")


@pytest.mark.parametrize("parts", [1, 2, 4])
def test_copy_pool_runs_every_part_once(tmp_path, parts):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    src = tmp_path / "pool_test.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "pool_test"
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(parts)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_copy_pool_default_parts_from_environment(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    src = tmp_path / "pool_env.cpp"
    src.write_text('#include "copy_pool.h"\n#include <cstdio>\nint main() { printf("%d\\n", CopyPool::default_parts()); }\n')
    exe = tmp_path / "pool_env"
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", "-I", CSRC, str(src), "-o", str(exe)], check=True)
    for val, expect in (("3", 3), ("1", 1), ("0", 1), ("500", 64)):
        r = subprocess.run([str(exe)], capture_output=True, text=True, env={**os.environ, "NB6_COPY_THREADS": val})
        assert int(r.stdout) == expect
    env = {k: v for k, v in os.environ.items() if k != "NB6_COPY_THREADS"}
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
    assert 1 <= int(r.stdout) <= 4
