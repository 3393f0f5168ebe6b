"""The host worker pool and the asynchronous copier of hyalite_b200/csrc/host_threads.h, built with
the host compiler and run on the CPU (tests/host_threads_test.cpp)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "hyalite_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_pool_and_copier(tmp_path):
    exe = tmp_path / "host_threads_test"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, os.path.join(HERE, "host_threads_test.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "OK", r.stdout + r.stderr
