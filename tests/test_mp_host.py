"""The multiprecision helpers of the kernels (blocksvibe_b200/csrc/mp.cuh) compiled for the host with g++
(tests/mp_host_check.cpp): the pole step's truncated product scan stays within its stated error bound,
round_safe never accepts an approximation whose rounding could differ from the exact sum's (planted
near-midpoint magnitudes, errors up to the bound), and add_norm_col, the moments kernel's addition with one
operand in shared memory, equals add_norm bit for bit."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "blocksvibe_b200", "csrc")


@pytest.fixture(scope="module")
def report(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("mp") / "mp_host_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, "-o", exe, os.path.join(HERE, "mp_host_check.cpp")],
                   check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True, timeout=600).stdout
    return {name: (int(n), int(bad)) for name, n, bad in (line.split() for line in out.strip().splitlines())}


@pytest.mark.parametrize("check", ["mac10", "mac34"])
def test_truncated_product_scan_within_bound(report, check):
    n, bad = report[check]
    assert n > 0 and bad == 0


@pytest.mark.parametrize("check", ["safe4", "safe10"])
def test_round_safe_is_sound(report, check):
    accepted, bad = report[check]
    assert accepted > 1000 and bad == 0


@pytest.mark.parametrize("check", ["col10", "col34", "col42"])
def test_add_norm_col_equals_add_norm(report, check):
    n, bad = report[check]
    assert n > 0 and bad == 0
