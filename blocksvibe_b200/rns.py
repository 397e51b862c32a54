"""Host side of the residue-number-system GEMM (csrc/rns.cuh): prime tables per limb count and the three
launches (digit split, tensor-core residue product, CRT).  ``gemm_rns(A, B)`` has the semantics of
``mpf.gemm`` and returns the same bits as the schoolbook path: both compute the exact integer dot products
of the aligned operands and round once."""
import ctypes
from math import prod

import numpy as np
import torch

from . import _lib
from .mpf import MPF, align_cols, align_rows

_P = ctypes.c_void_p
_I = ctypes.c_int
_Q = ctypes.c_int64


class RnsTables(ctypes.Structure):
    _fields_ = [("p", _P), ("mu", _P), ("w", _P), ("conv", _P), ("inv", _P), ("mj", _P), ("mfull", _P),
                ("np", _I), ("ml", _I), ("mtop", ctypes.c_uint64), ("msw", _I)]


class RnsMmaArgs(ctypes.Structure):
    _fields_ = [("X", _P), ("Y", _P), ("x_mat", _Q), ("y_mat", _Q), ("nb", _Q), ("NI", _Q), ("NL", _Q),
                ("Kp", _I), ("TN", _I), ("tiles_l", _Q), ("out_b", _Q), ("out_i", _Q), ("out_l", _Q),
                ("out", _P), ("err", _P), ("yb", _P), ("crt_kp", _Q)]


class RnsSplitArgs(ctypes.Structure):
    _fields_ = [("m", _P), ("plane", _Q), ("nb", _Q), ("R", _Q), ("K", _Q), ("sb", _Q), ("sr", _Q), ("sk", _Q),
                ("Rp", _Q), ("Kp", _Q), ("TR", _I), ("mat_bytes", _Q), ("out", _P), ("C", _P), ("Ks", _I), ("NS", _I),
                ("err", _P)]


class RnsCrtArgs(ctypes.Structure):
    _fields_ = [("A", _P), ("T", _P), ("Kc", _I), ("NH", _I), ("n", _Q), ("nbatch", _Q), ("M", _Q), ("N", _Q),
                ("ea", _P), ("eb", _P), ("cm", _P), ("ce", _P), ("cplane", _Q), ("err", _P)]


def _bind():
    lib = _lib.lib()
    if getattr(lib, "_rns_bound", False):
        return lib
    lib.b3d_rns_layout.argtypes = [_I, ctypes.POINTER(_I), ctypes.POINTER(_I)]
    lib.b3d_rns_split.argtypes = [_I, _P, _Q, _Q, _Q, _Q, _Q, _Q, _Q, _Q, _Q, _I, ctypes.POINTER(RnsTables), _P, _Q, _P]
    lib.b3d_rns_mma.argtypes = [ctypes.POINTER(RnsMmaArgs), ctypes.POINTER(RnsTables), _P]
    lib.b3d_rns_crt.argtypes = [_I, _P, _Q, _P, _P, _Q, _Q, _Q, ctypes.POINTER(RnsTables), _P, _P, _Q, _P]
    lib.b3d_rns_crt_mma.argtypes = [_I, ctypes.POINTER(RnsCrtArgs), ctypes.POINTER(RnsTables), _P]
    lib.b3d_rns_split_mma.argtypes = [_I, ctypes.POINTER(RnsSplitArgs), ctypes.POINTER(RnsTables), _P]
    for f in (lib.b3d_rns_layout, lib.b3d_rns_split, lib.b3d_rns_mma, lib.b3d_rns_crt, lib.b3d_rns_crt_mma,
              lib.b3d_rns_split_mma):
        f.restype = _I
    lib._rns_bound = True
    return lib


def _check(rc, name):
    if rc != 0:
        raise _lib.B3DError(f"{name} failed ({rc}): {_lib.lib().b3d_last_error().decode()}")


def _is_prime(n):
    """deterministic Miller-Rabin for n < 2^64"""
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def primes_below_2_31(count):
    out, n = [], (1 << 31) - 1
    while len(out) < count:
        if _is_prime(n):
            out.append(n)
        n -= 2
    return out


def layout(L):
    lib = _bind()
    np_, ml = _I(), _I()
    _check(lib.b3d_rns_layout(L, ctypes.byref(np_), ctypes.byref(ml)), "b3d_rns_layout")
    return np_.value, ml.value


def crt_quotient_words(M):
    """(msw, mtop) of the integer CRT quotient (csrc/rns.cuh crt_quotient): the least word offset with
    32 msw >= bitlen(M) - 56, and floor(M / 2^(32 msw))"""
    msw = max(0, -(-(M.bit_length() - 56) // 32))
    return msw, M >> (32 * msw)


def crt_quotient(xp, msw, mtop):
    """the kernels' quotient: round(xt / mtop) by seven compare-and-add steps, xt = words msw, msw + 1 of x'"""
    xt = (xp >> (32 * msw)) & ((1 << 64) - 1)
    num, den = 2 * xt + mtop, 2 * mtop
    assert num < 1 << 64
    q = 0
    for b in range(6, -1, -1):
        if (q + (1 << b)) * den <= num:
            q += 1 << b
    return q


class Tables:
    """constant tables for L-limb operands on one device"""

    def __init__(self, L, device):
        self.L = L
        npr, ml = layout(L)
        ps = primes_below_2_31(npr)
        M = prod(ps)
        NB = 32 * L - 2
        assert M.bit_length() > 2 * NB + 12 + 2, "prime set too small"
        assert M.bit_length() <= 32 * ml
        limbs = lambda x, n: [(x >> (32 * i)) & 0xFFFFFFFF for i in range(n)]
        mj = [M // p for p in ps]
        t = lambda a, dt: torch.tensor(np.array(a, dtype=dt), device=device)
        self.p = t(ps, np.uint32).view(torch.int32)
        self.mu = t([(1 << 62) // p for p in ps], np.uint64).view(torch.int64)
        self.w = t([[pow(2, 8 * u, p) for u in range(8)] for p in ps], np.uint32).view(torch.int32)
        self.conv = t([[pow(2, 32 * k, p) for k in range(L)] for p in ps], np.uint32).view(torch.int32)
        self.inv = t([pow(m % p, -1, p) for m, p in zip(mj, ps)], np.uint32).view(torch.int32)
        self.mj = t([limbs(m, ml) for m in mj], np.uint32).view(torch.int32)
        self.mfull = t(limbs(M, ml), np.uint32).view(torch.int32)
        self.msw, self.mtop = crt_quotient_words(M)
        self.np, self.ml = npr, ml
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        # CRT operand geometry and the constant Toeplitz digits T[pos][4 j + a] = byte (pos - a) of M / p_j
        self.Kc = _round_up(4 * npr, 32)
        P = 4 * ml + 3
        self.NH = _round_up(-(-P // 2), 16)
        mb = np.array([limbs(m, ml) for m in mj], dtype=np.uint32).view(np.uint8).reshape(npr, 4 * ml)
        T = np.zeros((2 * self.NH, self.Kc), dtype=np.uint8)
        for jj in range(npr):
            for a in range(4):
                T[a:a + 4 * ml, 4 * jj + a] = mb[jj]
        tiles = [T[h * self.NH:(h + 1) * self.NH].reshape(self.NH // 8, 8, self.Kc // 16, 16).transpose(2, 0, 1, 3)
                 for h in range(2)]
        self.T = torch.from_numpy(np.ascontiguousarray(np.concatenate([t.reshape(-1) for t in tiles]))).to(device)
        # split constants C[(j, t)][d] = byte t of (2^(8 d) mod p_j), d < 4 L: the magnitude bytes times C give
        # the residues' byte-weighted sums
        self.Ks = _round_up(4 * L, 32)
        self.NS = _round_up(-(-4 * npr // 2), 16)
        C = np.zeros((2 * self.NS, self.Ks), dtype=np.uint8)
        for jj, p in enumerate(ps):
            for d in range(4 * L):
                v = pow(2, 8 * d, p)
                for t4 in range(4):
                    C[4 * jj + t4, d] = (v >> (8 * t4)) & 0xFF
        tiles = [C[h * self.NS:(h + 1) * self.NS].reshape(self.NS // 8, 8, self.Ks // 16, 16).transpose(2, 0, 1, 3)
                 for h in range(2)]
        self.C = torch.from_numpy(np.ascontiguousarray(np.concatenate([t.reshape(-1) for t in tiles]))).to(device)
        self.c = RnsTables(self.p.data_ptr(), self.mu.data_ptr(), self.w.data_ptr(), self.conv.data_ptr(),
                           self.inv.data_ptr(), self.mj.data_ptr(), self.mfull.data_ptr(), npr, ml, self.mtop,
                           self.msw)


_TABLES = {}


def tables(L, device):
    key = (L, str(device))
    if key not in _TABLES:
        _TABLES[key] = Tables(L, device)
    return _TABLES[key]


def _round_up(x, m):
    return -(-x // m) * m


SPLIT = "tensor"          # "tensor": residue digits on the tensor cores; "cuda": on the CUDA cores

# int8 multiply-accumulates issued to the tensor cores by the residue products since the last reset (the work
# of k_rns_mma: 128 x TN x Kp per CTA), for the INT8 roofline
MMA_STATS = {"macs": 0, "alg_macs": 0, "calls": 0}
MMA_TIMER = None          # a list: (start, end) CUDA events are appended around every tensor-core product launch


def _split(tb, m, plane, nb, R, K, sb, sr, sk, Kp, TR, stream):
    """digit matrices (np, nb, 4 Rp x Kp) of an aligned operand with R rows, tiles of TR digit rows"""
    rows_per_tile = TR // 4
    Rp = _round_up(max(R, 1), rows_per_tile)
    mat = 4 * Rp * Kp
    out = torch.empty(tb.np * nb * mat, dtype=torch.uint8, device=m.device)
    if SPLIT == "tensor":
        args = RnsSplitArgs(m.data_ptr(), plane, nb, R, K, sb, sr, sk, Rp, Kp, TR, mat, out.data_ptr(),
                            tb.C.data_ptr(), tb.Ks, tb.NS, tb.err.data_ptr())
        _check(_bind().b3d_rns_split_mma(tb.L, ctypes.byref(args), ctypes.byref(tb.c), stream), "b3d_rns_split_mma")
    else:
        _check(_bind().b3d_rns_split(tb.L, m.data_ptr(), plane, nb, R, K, sb, sr, sk, Rp, Kp, TR, ctypes.byref(tb.c),
                                     out.data_ptr(), mat, stream), "b3d_rns_split")
    return out, mat, Rp


def gemm_aligned_rns(Aal, Bal, crt="tensor", lanes=None):
    """(row-aligned A (L, nb, M, K), (nb, M)) x (column-aligned B (L, nb, K, N), (nb, N)) -> MPF (nb, M, N),
    on the tensor cores; K <= 256.  lanes: "a" or "b", the operand whose rows go on the 128 TMEM lanes
    (default: the one with more rows)"""
    am, ae = Aal
    bm, be = Bal
    L, nb, M, K = am.shape
    N = bm.shape[-1]
    dev = am.device
    if K > 256:
        raise ValueError("gemm_aligned_rns: K > 256")
    tb = tables(L, dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    Kp = _round_up(max(K, 1), 32)
    # the operand with more rows goes on the 128 TMEM lanes
    a_rows = dict(m=am, plane=am.stride(0), R=M, sb=M * K, sr=K, sk=1)
    b_rows = dict(m=bm, plane=bm.stride(0), R=N, sb=K * N, sr=1, sk=N)
    if (lanes is None and M >= N) or lanes == "a":
        xs, ys, out_i, out_l = a_rows, b_rows, N, 1
    else:
        xs, ys, out_i, out_l = b_rows, a_rows, 1, N
    NL = ys["R"]
    TN = min(256, _round_up(4 * NL, 16))
    X, x_mat, _ = _split(tb, xs["m"], xs["plane"], nb, xs["R"], K, xs["sb"], xs["sr"], xs["sk"], Kp, 128, stream)
    Y, y_mat, Rp_y = _split(tb, ys["m"], ys["plane"], nb, NL, K, ys["sb"], ys["sr"], ys["sk"], Kp, TN, stream)
    n = nb * M * N
    cm = torch.empty((L, n), dtype=torch.int32, device=dev)
    ce = torch.empty((nb, M, N), dtype=torch.int64, device=dev)
    ae, be = ae.contiguous(), be.contiguous()
    MMA_STATS["macs"] += tb.np * nb * (x_mat // Kp) * TN * (4 * Rp_y // TN) * Kp
    MMA_STATS["alg_macs"] += tb.np * nb * M * N * K * 16         # 4 x 4 byte products per residue product
    MMA_STATS["calls"] += 1
    if crt == "tensor":                                     # y bytes -> CRT on the tensor cores
        # padding columns of the y bytes meet zero rows of the constant matrix T, padding rows are never stored
        yb = torch.empty(_round_up(max(n, 1), 128) * tb.Kc, dtype=torch.uint8, device=dev)
        args = RnsMmaArgs(X.data_ptr(), Y.data_ptr(), x_mat, y_mat, nb, xs["R"], NL, Kp, TN, (4 * Rp_y) // TN,
                          M * N, out_i, out_l, None, tb.err.data_ptr(), yb.data_ptr(), tb.Kc)
        if MMA_TIMER is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        _check(_bind().b3d_rns_mma(ctypes.byref(args), ctypes.byref(tb.c), stream), "b3d_rns_mma")
        if MMA_TIMER is not None:
            ev[1].record()
            MMA_TIMER.append(ev)
        cargs = RnsCrtArgs(yb.data_ptr(), tb.T.data_ptr(), tb.Kc, tb.NH, n, nb, M, N, ae.data_ptr(), be.data_ptr(),
                           cm.data_ptr(), ce.data_ptr(), cm.stride(0), tb.err.data_ptr())
        _check(_bind().b3d_rns_crt_mma(L, ctypes.byref(cargs), ctypes.byref(tb.c), stream), "b3d_rns_crt_mma")
    else:                                                   # residues -> CRT on the CUDA cores
        res = torch.empty(tb.np * n, dtype=torch.int32, device=dev)
        args = RnsMmaArgs(X.data_ptr(), Y.data_ptr(), x_mat, y_mat, nb, xs["R"], NL, Kp, TN, (4 * Rp_y) // TN,
                          M * N, out_i, out_l, res.data_ptr(), tb.err.data_ptr(), None, 0)
        _check(_bind().b3d_rns_mma(ctypes.byref(args), ctypes.byref(tb.c), stream), "b3d_rns_mma")
        _check(_bind().b3d_rns_crt(L, res.data_ptr(), n, ae.data_ptr(), be.data_ptr(), nb, M, N, ctypes.byref(tb.c),
                                   cm.data_ptr(), ce.data_ptr(), cm.stride(0), stream), "b3d_rns_crt")
    return MPF(cm.reshape(L, nb, M, N), ce)


def check_errors(device):
    """raise if a tensor-core launch on `device` recorded a timeout (bounded mbarrier waits)"""
    for (L, dev), tb in _TABLES.items():
        if dev == str(device) and int(tb.err.item()) != 0:
            code = int(tb.err.item())
            tb.err.zero_()
            raise _lib.B3DError(f"b3d_rns_mma: a wait timed out (code {code})")
