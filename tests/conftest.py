import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libb3dgpu.so")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def golden_operator(case):
    """M dict (key -> matrix of strings) and h_inf entries of a golden recursion case"""
    M = {((P[0], P[1]), d, tjnn, ppq, tj): mat for P, d, tjnn, ppq, tj, mat in case["M"]}
    return M, case["h_inf"]


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
