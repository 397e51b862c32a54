"""Index plan of the batched radial recursion for one operator, built by the library's host C++ builder
(``b3d_plan_build``, csrc/plan.cpp) and held here as numpy arrays.  Host half of the reference's
``recursion_gpu.Plan`` (``blocksvibe/recursion_gpu.py:136-365``): same constructor arguments and attribute
names, the same tensors (golden plans of the reference pin them bit for bit).

The recursion of blocks_3d (fill_residues.cxx) computes, level by level in m, one residue block per (parity p,
spin tj, pole P); the operator does not depend on the right-hand side, so its whole index structure is built once:

* a logical slot per residue block, ``p * nslots + first(m, spin index) + pole index``;
* per level, the Cauchy groups (src, tj'), their rows (distinct D') and columns (the prime poles of tj' at
  order m and the slots holding them): ``gsrc, gj, rowd, nrow, cold, ncol, col``;
* per pole-step task: output slot, H row, L / R matrix keys, Q key, (L, Q) pair, and the task itself
  (parity, spin, pole kind and k): ``t_slot, t_hrow, t_L, t_R, t_q, t_qL, t_p, t_tj, t_kind, t_k``;
* with ``reuse=True`` a physical slot per logical one, recycled after the last level that reads it.
"""
import ctypes

import numpy as np

from . import _lib

LEVEL_FIELDS = ("gsrc", "gj", "col", "rowd", "nrow", "cold", "ncol",
                "t_slot", "t_hrow", "t_L", "t_R", "t_q", "t_qL", "t_p", "t_tj", "t_kind", "t_k")


class _LevelArrays(ctypes.Structure):
    """struct b3d_plan_level_arrays"""
    _fields_ = [(f, ctypes.c_void_p) for f in LEVEL_FIELDS]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Plan:
    """Index plan for (two_j12, two_j43, two_j_max, order, pseudo_parities); levels without any task are None."""

    def __init__(self, two_j12, two_j43, two_j_max, order, pseudo_parities, reuse=False):
        self.tj12, self.tj43, self.tjmax, self.order = two_j12, two_j43, two_j_max, order
        self.pp = tuple(tuple(int(v) for v in x) for x in pseudo_parities)
        self.base = two_j12 % 2
        lib = _lib.lib()
        handle = ctypes.c_void_p()
        pp = np.array(self.pp, dtype=np.int64).reshape(4)
        _lib.call("b3d_plan_build", two_j12, two_j43, two_j_max, order, _ptr(pp), int(bool(reuse)), ctypes.byref(handle))
        try:
            self._copy_out(handle)
        finally:
            lib.b3d_plan_destroy(handle)

    def _copy_out(self, h):
        sc = np.zeros(11, dtype=np.int64)
        _lib.call("b3d_plan_scalars", h, _ptr(sc))
        (self.Smax, self.Jh, self.nslots, self.nphys, self.zero_slot, self.dmax, _, nM, nQ, nLQ, nlay) = (int(x) for x in sc)
        mk, qk, lq = np.zeros((nM, 5), np.int64), np.zeros((nQ, 4), np.int64), np.zeros((nLQ, 2), np.int64)
        _lib.call("b3d_plan_keys", h, _ptr(mk), _ptr(qk), _ptr(lq))
        self.Mkeys = {((a, b), side, self.tj12 if side == 0 else self.tj43, ppq, tj): i
                      for i, (a, b, side, ppq, tj) in enumerate(mk.tolist())}
        self.Qkeys = {((a, b), tj, sign): i for i, (a, b, tj, sign) in enumerate(qk.tolist())}
        self.LQpairs = lq
        self._start, self._first = np.zeros(self.order, np.int64), np.zeros(nlay, np.int64)
        self.phys = np.zeros(2 * self.nslots, np.int64)
        _lib.call("b3d_plan_layout", h, _ptr(self._start), _ptr(self._first), _ptr(self.phys))
        self.levels = []
        dims = np.zeros(4, np.int64)
        for m in range(self.order):
            _lib.call("b3d_plan_level_dims", h, m, _ptr(dims))
            nb, Mr, Kc, T = (int(x) for x in dims)
            if nb == 0:
                self.levels.append(None)
                continue
            shape = dict(gsrc=nb, gj=nb, nrow=nb, ncol=nb, rowd=(nb, Mr), col=(nb, Kc), cold=(nb, Kc))
            lev = {f: np.zeros(shape.get(f, T), np.int64) for f in LEVEL_FIELDS}
            arr = _LevelArrays(**{f: _ptr(lev[f]).value for f in LEVEL_FIELDS})
            _lib.call("b3d_plan_level", h, m, ctypes.byref(arr))
            lev.update(m=m, nb=nb, Mr=Mr, Kc=Kc)
            self.levels.append(lev)

    def offset(self, m, jidx):
        """first logical slot of spin index jidx at level m (parity 0)"""
        return int(self._first[self._start[m] + jidx])

    def phys_slots(self, logical):
        """physical slots of logical ones (the zero slot where never written)"""
        logical = np.asarray(logical, dtype=np.int64)
        inside = logical < len(self.phys)
        p = self.phys[np.where(inside, logical, 0)]
        return np.where(inside & (p >= 0), p, self.zero_slot)

    def phys_slot(self, logical):
        return int(self.phys_slots(np.array([logical]))[0])

    def counts(self):
        """(Cauchy output entries, pole-step output entries) per right-hand side, rows padded per level and
        structures padded to Smax^2 (reference ``recursion_gpu.py:360``)"""
        s2 = self.Smax ** 2
        h = sum(lev["nb"] * lev["Mr"] for lev in self.levels if lev) * s2
        r = sum(len(lev["t_slot"]) for lev in self.levels if lev) * s2
        return h, r


def cauchy_tables(lev):
    """dense Cauchy tables of a level from its row / column pole positions: cdiff[g, r, i] = D'_r - D_i (0 on
    padding rows / columns and where the positions coincide) and cidx, the entry of the +-2/k table
    (0: zero, 2k - 1: +2/k, 2k: -2/k) (reference ``recursion_gpu.py:368-376``)"""
    nb, Mr, Kc = lev["nb"], lev["Mr"], lev["Kc"]
    cdiff = np.zeros((nb, Mr, Kc), dtype=np.int64)
    for g in range(nb):
        r, c = int(lev["nrow"][g]), int(lev["ncol"][g])
        cdiff[g, :r, :c] = np.subtract.outer(lev["rowd"][g, :r], lev["cold"][g, :c])
    cidx = 2 * np.abs(cdiff) - (cdiff > 0)
    cidx[cdiff == 0] = 0
    return cdiff.astype(np.int32), cidx
