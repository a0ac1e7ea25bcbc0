"""The scan's host thread pool (csrc/host_pool.hpp), compiled with the host compiler and
run on the CPU: exactly-once execution over many rounds and exception delivery."""

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_host_pool_runs_every_task_once(tmp_path):
    exe = tmp_path / "host_pool_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", str(ROOT / "solprop_b200" / "csrc"),
                    str(ROOT / "tests" / "host_pool_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "ok"
