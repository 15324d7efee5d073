"""The record staging plan of the FP32C staged kernels, checked on the CPU:
a small C++ program built from the plan header simulates the staging copies
for random stencil slices and checks every lane's staged read."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_stage_plan_lane_reads(tmp_path):
    exe = tmp_path / "stage_plan_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(exe), os.path.join(HERE, "native", "stage_plan_check.cpp")],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ")
