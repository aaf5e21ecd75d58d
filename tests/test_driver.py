"""The init/step/output driver (mhd_run_case) and the run-comparison tool.

CPU: the comparison tool's pass rule and exit codes (the reference's
scripts/compare_runs.py contract).  GPU: the driver's CSVs for the reference's
Brio-Wu case equal the oracle's, character for character; the device-resident
loop, FP32-bulk and device initial data agree within their tolerances.
"""
import os
import subprocess

import numpy as np
import pytest

from mhd_gpu_acc_b200 import F32, F64, Grid2DGPU, get_n_case_config, initialise, load
from mhd_gpu_acc_b200.compare import compare

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "mhd_gpu_acc_b200", "mhd_run_case")


def _write(d, name, arr):
    os.makedirs(d, exist_ok=True)
    np.savetxt(os.path.join(d, name), arr, delimiter=",", fmt="%.8e")


def test_compare_pass_fail_and_exit_codes(tmp_path):
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    x = np.linspace(1, 2, 12).reshape(3, 4)
    _write(a, "case_gpu_t10_rho.csv", x)
    _write(b, "case_gpu_t10_rho.csv", x * (1 + 1e-7))
    _write(a, "case_gpu_t10_p.csv", x)
    _write(b, "case_gpu_t10_p.csv", x + 1e-3)
    out = open(os.devnull, "w")
    assert compare(a, b, fields=["rho"], out=out) == 0       # max_rel 1e-7 <= 1e-6
    assert compare(a, b, out=out) == 1                       # p fails both tolerances
    assert compare(a, b, tol=1e-2, out=out) == 0
    assert compare(a, str(tmp_path / "empty"), out=out) == 2
    _write(b, "case_gpu_t10_v.csv", x[:2])
    _write(a, "case_gpu_t10_v.csv", x)
    assert compare(a, b, fields=["v"], out=out) == 2         # shape mismatch


def _csv(field):
    return "".join(",".join("%.8e" % v for v in row) + "\n" for row in field[::-1])


def _run(args, cwd):
    r = subprocess.run([DRIVER, *args], capture_output=True, text=True, timeout=600, cwd=cwd)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.mark.gpu
def test_driver_brio_wu_csv_equals_oracle(oracle, tmp_path):
    cfg = get_n_case_config(2, 1)
    out = _run(["brio_wu", "--solver", "hllc", "--out", str(tmp_path / "g")], str(tmp_path))
    bc = (cfg.bc.left, cfg.bc.right, cfg.bc.bottom, cfg.bc.top)
    U0 = initialise(2, cfg.nx, cfg.ny, 2, cfg.extent)
    rc, U, t, steps, ch, _ = oracle.run(U0, 2, cfg.dx, cfg.dy, cfg.gamma, cfg.cfl, 1, 0, bc, t_end=cfg.t_end)
    assert f"steps={steps}" in out
    I = U[:, 2:-2, 2:-2]
    with open(tmp_path / "g" / "brio_wu_gpu_t10_rho.csv") as f:
        assert f.read() == _csv(I[0])
    with open(tmp_path / "g" / "brio_wu_gpu_t10_By.csv") as f:
        assert f.read() == _csv(I[5])


@pytest.mark.gpu
def test_driver_device_loop_and_fp32(tmp_path):
    _run(["shock_bubble_mhd", "--out", str(tmp_path / "host")], str(tmp_path))
    _run(["shock_bubble_mhd", "--device-loop", "--out", str(tmp_path / "dev")], str(tmp_path))
    _run(["shock_bubble_mhd", "--device-loop", "--device-ic", "--precision", "fp32", "--out",
          str(tmp_path / "f32")], str(tmp_path))
    devnull = open(os.devnull, "w")
    # device-resident dt (device exp for the damping factor): rounding-level agreement
    assert compare(str(tmp_path / "host"), str(tmp_path / "dev"), tol=1e-9, rtol=1e-9, out=devnull) == 0
    # FP32-bulk against FP64: shock positions may shift by a cell, so compare the
    # density in relative L1 (<= 1e-4 for this Mach-10 run to t_end)
    a = np.loadtxt(tmp_path / "host" / "shock_bubble_mhd_gpu_t6_rho.csv", delimiter=",")
    b = np.loadtxt(tmp_path / "f32" / "shock_bubble_mhd_gpu_t6_rho.csv", delimiter=",")
    assert np.abs(a - b).sum() / np.abs(a).sum() <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1, 2, 3, 4, 5])
def test_device_initial_data_matches_host(case):
    cfg = get_n_case_config(case, 1)
    nx, ny = min(cfg.nx, 96), min(cfg.ny, 64)
    ext = cfg.extent
    host = initialise(case, nx, ny, 2, ext)
    for dt, tol in ((F64, 1e-13), (F32, 1e-6)):
        g = Grid2DGPU(nx, ny, 2, *ext, dt)
        import ctypes as C

        assert load().mhd_initialise_device(None, C.byref(g.g), case) == 0
        got = g.download()
        scale = np.maximum(np.abs(host), 1.0)
        assert np.max(np.abs(got - host) / scale) <= tol, (case, dt)
