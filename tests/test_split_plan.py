"""The batched split planner stays inside the buffers sized for it (no GPU).

batch_plan / batch_max_split (starlab_b200/csrc/kernels.h) decide, per
call or cluster, how its j-range is cut into tasks; the batched kernels then
write split partials to part[split * ni + i], and the ensemble allocates
n * batch_max_split(nj_pad, min_tiles) records per cluster.  tests/plan_check.cu
includes the header itself, runs the planner on the host over every layout,
lane shape, tasks-wanted and fewest-tiles setting and i/j counts up to 2^18,
and checks each plan's bounds and coverage.
"""
import os
import shutil
import subprocess

import pytest

from starlab_b200 import build

HERE = os.path.dirname(os.path.abspath(__file__))


def test_batch_plans_stay_inside_their_partial_buffers(tmp_path):
    nvcc = build.NVCC if os.path.exists(build.NVCC) else shutil.which("nvcc")
    if not nvcc:
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "plan_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets",
                    "-I" + os.path.join(build.PKG, "csrc"), "-I" + os.path.join(build.REPO, "include"),
                    "-o", exe, os.path.join(HERE, "plan_check.cu")], check=True, capture_output=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.startswith("ok "), out.stdout + out.stderr
    assert int(out.stdout.split()[1]) > 100000
