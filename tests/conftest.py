import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on the B200 box)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import ORACLE_SO, Oracle, build

    if not os.path.exists(ORACLE_SO):
        build(ref=False)
    o = Oracle()
    o.set_threads(min(8, os.cpu_count() or 1))
    return o


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import REF_SO, Reference

    if not os.path.exists(REF_SO):
        pytest.skip("reference build oracle/_ref/libmhdref.so not present")
    r = Reference()
    r.set_threads(min(8, os.cpu_count() or 1))
    return r


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        runs = json.load(f)
    states = dict(np.load(os.path.join(GOLDEN, "states.npz")))
    return runs, states


@pytest.fixture(scope="session")
def lib():
    from mhd_gpu_acc_b200 import load

    return load()
