"""The serving loop's scheduling policy (csrc/scheduler.h), compiled with the
host C++ compiler and driven without a GPU: admission by memory budget,
passing over busy diagrams, eviction of the least recently used idle diagram
into the reuse pool, grouping of new diagrams, failures."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "integer_delauney_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_scheduler_policy(tmp_path):
    exe = str(tmp_path / "scheduler_host_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", CSRC,
                    os.path.join(HERE, "scheduler_host_test.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    assert "all checks passed" in out.stdout
    # the Python layer's budget figures equal the scheduler's
    from integer_delauney_b200.serving import estimate_bytes, slot_reserve
    for line in out.stdout.splitlines():
        f = line.split()
        if f[0] == "slot_reserve":
            assert slot_reserve(int(f[1])) == int(f[2])
        elif f[0] == "fresh":
            W, H, n, P, want = map(int, f[1:])
            assert estimate_bytes(W, H, n, P, workspace=False) == want
