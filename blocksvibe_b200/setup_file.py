"""b3d_setup's B3DSETUP file on the host: the input of the drop-in (the M matrices of a group and h_infinity per
four-point structure and lambda order, computed by blocks_3d's own setup code, csrc/b3d_setup.cxx of the
reference).  Host half of the reference's ``setup.read`` / ``MTable`` / ``h_inf_tensor``
(``blocksvibe/setup.py:77-180``): the numbers are rounded to the drop-in's limb count by the library
(``b3d_setup_numbers``) and kept in host memory until a plan asks for them.

Layout (``b3d_setup.cxx:15-21``; little-endian int64 words, K = limbs per number):

    "B3DSETUP" K
    nM; nM x [pole kind, k, side (0 = j12, 1 = j43), two_jNN, prime pseudo-parity, two_j, rows, cols];
        then every matrix entry, row-major, as a number
    ntasks; per task: q4[4] sign pp00 pp01 pp10 pp11 nn; per lambda order: n count;
        count x [parity, m, j, a, b]; count numbers
    number = [size exp limb_0 .. limb_{K-1}] (GMP mpf: 64-bit limbs, value
             sign(size) sum_t limb_t 2^(64 t) 2^(64 (exp - K)))

``write`` produces the same layout from exact numbers (for tests and synthetic inputs).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .mpf import EZ, MPF

MAGIC = np.frombuffer(b"B3DSETUP", dtype=np.int64)[0]


def _numbers(rec, K, L):
    """(n, 2 + K) int64 records -> host (m (L, n) int32, e (n,) int64)"""
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    n = rec.shape[0]
    m, e = np.zeros((L, n), np.int32), np.full(n, EZ, np.int64)
    if n:
        vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        _lib.call("b3d_setup_numbers", vp(rec), n, K, L, vp(m), n, vp(e))
    return m, e


class MTable:
    """M matrices of a setup file: hdr (nM, 8) int64 and their entries (host limbs), index[key] -> record with
    key = ((kind, k), side, two_jNN, pseudo-parity, two_j) (the plan's Mkeys convention)"""

    def __init__(self, hdr, m, e):
        self.hdr, self.m, self.e = hdr, m, e
        self.index = {((int(h[0]), int(h[1])), int(h[2]), int(h[3]), int(h[4]), int(h[5])): i
                      for i, h in enumerate(hdr)}
        cnt = hdr[:, 6] * hdr[:, 7]
        self.first = np.cumsum(cnt) - cnt

    @property
    def L(self):
        return self.m.shape[0]

    def for_plan(self, plan, device=None):
        """MPF (len(plan.Mkeys), Smax, Smax) in plan.Mkeys order (zero where the file has no matrix)"""
        Sm, nM = plan.Smax, len(plan.Mkeys)
        dst, src = [], []
        for key, i in plan.Mkeys.items():
            r = self.index.get(key)
            if r is None:
                continue
            rows, cols = int(self.hdr[r, 6]), int(self.hdr[r, 7])
            if rows > Sm or cols > Sm:
                raise ValueError(f"M matrix {key} is {rows} x {cols}, more than Smax = {Sm}")
            a, b = np.divmod(np.arange(rows * cols), cols)
            dst.append((i * Sm + a) * Sm + b)
            src.append(self.first[r] + np.arange(rows * cols))
        m = np.zeros((self.L, nM * Sm * Sm), np.int32)
        e = np.full(nM * Sm * Sm, EZ, np.int64)
        if dst:
            d, s = np.concatenate(dst), np.concatenate(src)
            m[:, d], e[d] = self.m[:, s], self.e[s]
        return MPF(torch.from_numpy(m).reshape(self.L, nM, Sm, Sm).to(device),
                   torch.from_numpy(e).reshape(nM, Sm, Sm).to(device))


class SetupTask:
    """one four-point structure of a setup file: q4 (doubled), sign, pseudo-parity types and, per lambda order n,
    h[n] = (index (count, 5) [parity, m, j, a, b], host limbs m (L, count), exponents e (count))"""

    def __init__(self, q4, sign, pp, h):
        self.q4, self.sign, self.pp, self.h = q4, sign, pp, h

    def h_inf(self, n, order, Jh, Smax):
        """MPF (2, order + 1, Jh, Smax^2) on the host: the layout of the recursion's h_inf for one lambda order
        (entries beyond order or Jh dropped, zeros elsewhere; reference setup.h_inf_tensor, setup.py:164-180)"""
        idx, m, e = self.h[n]
        L = m.shape[0]
        s, lev, j, a, b = idx.T
        ok = (lev <= order) & (j < Jh) & (a < Smax) & (b < Smax)
        flat = (((s * (order + 1) + lev) * Jh + j) * Smax + a) * Smax + b
        om = np.zeros((L, 2 * (order + 1) * Jh * Smax * Smax), np.int32)
        oe = np.full(om.shape[1], EZ, np.int64)
        om[:, flat[ok]], oe[flat[ok]] = m[:, ok], e[ok]
        shape = (2, order + 1, Jh, Smax * Smax)
        return MPF(torch.from_numpy(om).reshape((L,) + shape), torch.from_numpy(oe).reshape(shape))


def read(path, L, m_path=None):
    """(MTable, [SetupTask]) of a setup file with numbers at L limbs; the M matrices from m_path if given (a
    file written with the matrices only, as the reference's cache of them, setup.save_m)"""
    if m_path is not None:
        M, _ = read(m_path, L)
        _, tasks = read(path, L)
        return M, tasks
    raw = np.fromfile(path, dtype=np.int64)
    if len(raw) < 3 or raw[0] != MAGIC:
        raise ValueError(f"{path}: not a B3DSETUP file")
    K = int(raw[1])
    rl = 2 + K
    pos = 2

    def take(k):
        nonlocal pos
        if pos + k > len(raw):
            raise ValueError(f"{path}: truncated")
        out = raw[pos:pos + k]
        pos += k
        return out

    nM = int(take(1)[0])
    hdr = take(8 * nM).reshape(nM, 8).copy()
    nvals = int((hdr[:, 6] * hdr[:, 7]).sum())
    M = MTable(hdr, *_numbers(take(rl * nvals).reshape(nvals, rl), K, L))
    tasks = []
    for _ in range(int(take(1)[0])):
        t = take(10)
        q4, sign = tuple(int(x) for x in t[:4]), int(t[4])
        pp = ((int(t[5]), int(t[6])), (int(t[7]), int(t[8])))
        h = {}
        for _ in range(int(t[9])):
            n, cnt = (int(x) for x in take(2))
            idx = take(5 * cnt).reshape(cnt, 5).copy()
            h[n] = (idx,) + _numbers(take(rl * cnt).reshape(cnt, rl), K, L)
        tasks.append(SetupTask(q4, sign, pp, h))
    if pos != len(raw):
        raise ValueError(f"{path}: trailing data")
    return M, tasks


def _record(x, K):
    """[size, exp, limbs] of an exact number (mpmath or int), truncated toward zero to K 64-bit limbs as GMP's
    mpf holds it"""
    if isinstance(x, int):
        sign, man, ex, bc = x < 0, abs(x), 0, abs(x).bit_length()
    else:
        sign, man, ex, bc = x._mpf_                      # exact: never rounded to the working precision
    if not man:
        return [0, 0] + [0] * K
    top = ex + bc                                        # |x| < 2^top
    gexp = -(-top // 64)                                 # limbs above the radix point
    sh = ex + 64 * (K - gexp)
    mag = man << sh if sh >= 0 else man >> -sh
    limbs = [(mag >> (64 * t)) & ((1 << 64) - 1) for t in range(K)]
    words = [int(np.array(v, dtype=np.uint64).view(np.int64)) for v in limbs]
    return [-K if sign else K, gexp] + words


def write(path, K, matrices, tasks):
    """a B3DSETUP file: matrices {key ((kind, k), side, two_jNN, pp, two_j): list of rows of numbers};
    tasks [(q4, sign, pp, {n: [(parity, m, j, a, b, number)]})]"""
    w = [int(MAGIC), K, len(matrices)]
    vals = []
    for ((kind, k), side, tjnn, ppq, tj), rows in matrices.items():
        w += [kind, k, side, tjnn, ppq, tj, len(rows), len(rows[0]) if rows else 0]
        vals += [x for row in rows for x in row]
    for x in vals:
        w += _record(x, K)
    w.append(len(tasks))
    for q4, sign, pp, h in tasks:
        w += list(q4) + [sign, pp[0][0], pp[0][1], pp[1][0], pp[1][1], len(h)]
        for n, ents in h.items():
            w += [n, len(ents)]
            for ent in ents:
                w += list(ent[:5])
            for ent in ents:
                w += _record(ent[5], K)
    np.array(w, dtype=np.int64).tofile(path)
