"""The sweeps' task plans (x row segments, y row bands with guided sizes) cover
every cell of the grid exactly once, for extents from 1 to 5000 and every work
size the launches and the batch autotuner use.  The check is plain index
arithmetic compiled for the host (tests/plan_check.cu); it needs nvcc but no
GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="needs nvcc")
def test_sweep_plans_cover_every_cell_once(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "plan_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-x", "cu", "-Wno-deprecated-gpu-targets", "-I",
                    os.path.join(ROOT, "mhd_gpu_acc_b200", "csrc"), os.path.join(ROOT, "tests", "plan_check.cu"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "0 failures" in r.stdout
