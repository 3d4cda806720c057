"""The host copy pool of the banded host calls (hype-parallel_b200/csrc/hype_hostcopy.cu),
on the CPU: a small harness compiled with the pool's own source checks contiguous and
pitched copies against memcpy, copies issued from several threads at once, and a copy in a
forked child (which must start a pool of its own)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "hype-parallel_b200", "csrc")


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc to compile the pool's source")
def test_host_copy_pool(tmp_path):
    exe = tmp_path / "harness"
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", SRC, os.path.join(SRC, "hype_hostcopy.cu"),
                    os.path.join(ROOT, "tests", "host_copy", "harness.cpp"), "-o", str(exe), "-lpthread"],
                   check=True, capture_output=True, timeout=600)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
