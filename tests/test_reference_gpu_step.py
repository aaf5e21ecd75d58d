"""The reference's own GPU step (its src/gpu, compiled for sm_100a from the
reference sources by oracle/Makefile) and the B200 step behind the drop-in
headers, driven by the same host loop (oracle/gpu_step_timer.cu): both run the
reference's Orszag-Tang case, and the drop-in step is the faster one."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_timer")
OURS = os.path.join(ROOT, "oracle", "_ref", "dropin_gpu_timer")


def _time(exe, n, warmup, steps):
    r = subprocess.run([exe, str(n), str(warmup), str(steps)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.gpu
def test_dropin_step_outruns_the_reference_gpu_step():
    if not (os.path.exists(REF) and os.path.exists(OURS)):
        pytest.skip("oracle/_ref timers not built (make -C oracle timers)")
    ref = _time(REF, 8, 3, 20)
    ours = _time(OURS, 8, 3, 20)
    print(f"reference GPU step {ref['ms_per_step']:.3f} ms/step, drop-in B200 step {ours['ms_per_step']:.3f} ms/step "
          f"({ref['nx']}x{ref['ny']}, HLLD, FP64)")
    assert ref["nx"] == ours["nx"] == 1536
    assert ours["t"] > 0 and ref["t"] > 0
    assert ours["ms_per_step"] < ref["ms_per_step"]
