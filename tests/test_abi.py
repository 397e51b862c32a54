"""The C ABI library: it loads without a GPU and exports every entry point include/b3dgpu.h declares
(no compute calls here).  Host-side number conversions round-trip exactly.  CPU only."""
import os
import re
import subprocess

import mpmath as mp
import pytest
import torch

from conftest import ROOT
from blocksvibe_b200 import _lib, mpf


def _declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(b3d_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (b3d_\w+)", out))
    assert set(declared) <= exported
    assert set(_lib.exported_symbols()) <= exported


def test_library_metadata_calls():
    lib = _lib.lib()
    assert lib.b3d_version() >= 100
    for L in (6, 10, 14, 18, 22, 26, 30, 34, 38, 42, 46):
        assert lib.b3d_supported_limbs(L) == 1
    assert lib.b3d_supported_limbs(7) == 0


def test_limb_count_rule():
    """limbs(precision) of the reference's cli.py:270-274"""
    assert [mpf.limbs_for_precision(p) for p in (256, 512, 768, 896, 1024, 1280)] == [10, 18, 26, 30, 34, 42]


@pytest.mark.parametrize("L", [6, 10, 34])
def test_host_conversions_round_trip(L):
    mp.mp.prec = 32 * L + 64
    vals = [mp.mpf(0), mp.mpf(1), mp.mpf(-3) / 7, mp.pi * 2 ** 100, -mp.e * mp.mpf(2) ** -300, mp.mpf(2) ** 40 - 1]
    X = mpf.from_mp(vals, L)
    back = mpf.to_mp(X)
    NB = mpf.nbits(L)
    for v, b in zip(vals, back):
        assert abs(v - b) <= abs(v) * mp.mpf(2) ** (1 - NB)
    # normalised mantissas have exactly NB bits
    for man, e in mpf.to_ints(X):
        assert man == 0 or abs(man).bit_length() == NB
    # exact rationals
    from fractions import Fraction
    F = mpf.from_fractions([Fraction(1, 3), Fraction(-22, 7), Fraction(0)], L)
    got = mpf.to_mp(F)
    assert abs(got[0] - mp.mpf(1) / 3) < mp.mpf(2) ** (-NB)
    assert got[2] == 0


def test_kernels_refuse_cpu_tensors():
    X = mpf.zeros((3, 3), 10)
    with pytest.raises(_lib.B3DError):
        mpf.gemm(X, X)


def test_noalloc_refuses_oversized_batches_before_touching_the_device():
    """b3d_pole_level_noalloc checks T S^2 B (4 L + 8) against its fixed array factor by factor: a huge B (whose
    product with S^2 would wrap in 64 bits) and a huge T are refused with B3D_E_ARG before any CUDA call, so this
    runs without a GPU"""
    lib = _lib.lib()
    null = None
    for T, B, S in ((1, 1 << 52, 64), (1, (1 << 63) - 1, 64), (1 << 40, 1, 5), (2, 1 << 20, 5)):
        rc = lib.b3d_pole_level_noalloc(10, null, null, 0, null, null, 0, null, null, 0, null, null, null, null,
                                        T, B, S, null, null, 0, null)
        assert rc == -2, (T, B, S)
        assert b"scratch" in lib.b3d_last_error()
