"""Multiprecision floats on the GPU: the container, host conversions and the device operations.

An ``MPF`` holds ``m``, an int32 tensor of limb planes (L, *shape) (two's complement, limb 0 least
significant) and ``e``, an int64 tensor (*shape); the value of an element is m * 2^e.  Normalised values
have |m| of exactly NB = 32 L - 2 bits; zero is m = 0 with e = EZ.  This is the format the reference's
``sdpvibe.mpf.MPF`` exposes to blocksvibe (limb planes ``m``, exponents ``e``: reference
``cauchy.py:32``, ``derivatives.py:66,197``, ``b3djson.py:69-80``), so the drop-in boundary hands the
same arrays to the JSON writer.

Device operations (``gemm``, ``mul``, ``add``, ``align_rows``) call libb3dgpu.so through ctypes on the
current torch stream.  Host conversions round once to NB bits, half away from zero, as the device does.
"""
from math import prod

import mpmath as mp
import numpy as np
import torch
from mpmath import libmp

from . import _lib

EZ = -(1 << 60)


def nbits(L):
    return 32 * L - 2


def limbs_for_precision(precision):
    """GPU limbs for a blocks_3d precision: the precision rounded up to 64-bit words, plus 62 bits
    (reference ``cli.py:270-274``)"""
    rounded = ((precision - 1) // 64 + 1) * 64
    return -(-(rounded + 62) // 32)


class MPF:
    """limb planes m (L, *shape) int32 and exponents e (*shape) int64"""
    __slots__ = ("m", "e")

    def __init__(self, m, e):
        self.m, self.e = m, e

    @property
    def L(self):
        return self.m.shape[0]

    @property
    def shape(self):
        return tuple(self.e.shape)

    @property
    def device(self):
        return self.e.device

    def numel(self):
        return self.e.numel()

    def reshape(self, *shape):
        if len(shape) == 1 and isinstance(shape[0], (tuple, list)):
            shape = tuple(shape[0])
        return MPF(self.m.reshape(self.L, *shape), self.e.reshape(*shape))

    def permute(self, *perm):
        return MPF(self.m.permute(0, *[p + 1 for p in perm]), self.e.permute(*perm))

    def contiguous(self):
        return MPF(self.m.contiguous(), self.e.contiguous())

    def take(self, idx):
        """elements idx (any shape) along the first entry dimension"""
        return MPF(self.m[:, idx], self.e[idx])

    def __getitem__(self, key):
        key = key if isinstance(key, tuple) else (key,)
        return MPF(self.m[(slice(None),) + key], self.e[key])

    def expand(self, *shape):
        return MPF(self.m.expand(self.L, *shape), self.e.expand(*shape))

    def to(self, device):
        return MPF(self.m.to(device), self.e.to(device))

    def cpu(self):
        return self.to("cpu")


def zeros(shape, L, device=None):
    shape = tuple(shape)
    return MPF(torch.zeros((L,) + shape, dtype=torch.int32, device=device),
               torch.full(shape, EZ, dtype=torch.int64, device=device))


def cat(parts, dim):
    """concatenate along an entry dimension"""
    return MPF(torch.cat([p.m for p in parts], dim + 1), torch.cat([p.e for p in parts], dim))


# ---------------------------------------------------------------- host conversions

def _round(v, e, NB):
    """round the exact value v * 2^e (Python ints) to an NB-bit mantissa: (mantissa, exponent)"""
    if v == 0:
        return 0, EZ
    a = -v if v < 0 else v
    s = a.bit_length() - NB
    if s > 0:
        a = (a >> s) + ((a >> (s - 1)) & 1)
        if a.bit_length() > NB:
            a >>= 1
            s += 1
    elif s < 0:
        a <<= -s
    return (-a if v < 0 else a), e + s


def _pack(mants, exps, L, shape, device):
    n = len(mants)
    raw = b"".join(x.to_bytes(4 * L, "little", signed=True) for x in mants)
    m = np.frombuffer(raw, dtype=np.int32).reshape(n, L).T.copy() if n else np.zeros((L, 0), np.int32)
    shape = (n,) if shape is None else tuple(shape)
    return MPF(torch.from_numpy(m).reshape((L,) + shape).to(device),
               torch.tensor(exps, dtype=torch.int64).reshape(shape).to(device))


def from_ints(ints, exps, L, shape=None, device=None):
    """exact values ints[i] * 2^exps[i] rounded once to NB bits"""
    NB = nbits(L)
    out = [_round(int(v), int(e), NB) for v, e in zip(ints, exps)]
    return _pack([a for a, _ in out], [b for _, b in out], L, shape, device)


def from_fractions(fracs, L, shape=None, device=None):
    """exact rationals (fractions.Fraction or int) rounded to NB bits"""
    NB = nbits(L)
    out = []
    for f in fracs:
        num, den = int(f.numerator), int(f.denominator)
        if num == 0:
            out.append((0, EZ))
            continue
        a = abs(num)
        s = max(0, NB + 8 + den.bit_length() - a.bit_length())
        q = (a << s) // den                       # >= NB + 7 bits: truncation far below the rounding bit
        out.append(_round(-q if num < 0 else q, -s, NB))
    return _pack([a for a, _ in out], [b for _, b in out], L, shape, device)


def _mp_parts(x):
    """exact (mantissa, exponent) of an mpmath number or a Python int (never rounded to mpmath's
    working precision)"""
    if isinstance(x, int):
        return x, 0
    if not isinstance(x, mp.mpf):
        raise TypeError(f"expected an mpmath mpf or an int, got {type(x).__name__}")
    sign, man, exp, _ = x._mpf_
    if man == 0 and exp != 0:
        raise ValueError(f"not a finite number: {x}")
    return (-man if sign else man), exp


def from_mp(vals, L, shape=None, device=None):
    """mpmath numbers (or anything mp.mpf accepts exactly) rounded once to NB bits"""
    NB = nbits(L)
    out = [_round(*_mp_parts(x), NB) for x in vals]
    return _pack([a for a, _ in out], [b for _, b in out], L, shape, device)


def from_strings(strs, L, shape=None, device=None):
    """decimal strings, read at 32 L + 64 bits, then rounded to NB bits"""
    with mp.workprec(32 * L + 64):
        vals = [mp.mpf(s) for s in strs]
    return from_mp(vals, L, shape, device)


def to_ints(X):
    """list of exact (mantissa, exponent) pairs, flattened (zero: (0, EZ))"""
    m = X.m.detach().cpu().reshape(X.L, -1)
    e = X.e.detach().cpu().reshape(-1).tolist()
    raw = np.ascontiguousarray(m.numpy().T).view(np.uint8)
    return [(int.from_bytes(raw[i].tobytes(), "little", signed=True), e[i]) for i in range(len(e))]


def to_mp(X):
    """numpy object array of exact mpmath values with X's shape"""
    vals = [mp.make_mpf(libmp.from_man_exp(v, ex)) if v and ex != EZ else mp.mpf(0) for v, ex in to_ints(X)]
    out = np.empty(len(vals), dtype=object)
    out[:] = vals
    return out.reshape(X.shape)


# ---------------------------------------------------------------- device operations

def _stream(device):
    return ctypes_stream(torch.cuda.current_stream(device))


def ctypes_stream(s):
    return s.cuda_stream


def _check(*xs):
    for x in xs:
        if x.device.type != "cuda":
            raise _lib.B3DError("multiprecision kernels need CUDA tensors (no CPU path)")


def _ptr(t):
    return t.data_ptr() if t is not None else None


def align_rows(X, bidx=None, kmajor=False):
    """X: MPF (..., R, K).  Mantissas aligned to each row's largest exponent: (m (L, nb, R, K) or
    (L, nb, K, R) if kmajor, row exponents (nb, R)).  bidx: optional batch gather (rows of a table)."""
    _check(X)
    X = X.contiguous()
    R, K = X.shape[-2:]
    nt = prod(X.shape[:-2])
    nb = nt if bidx is None else bidx.numel()
    out = torch.empty((X.L, nb * R * K), dtype=torch.int32, device=X.device)
    oe = torch.empty((nb, R), dtype=torch.int64, device=X.device)
    if bidx is not None:
        bidx = bidx.reshape(-1).to(device=X.device, dtype=torch.int64).contiguous()
    _lib.call("b3d_align", X.L, _ptr(X.m), _ptr(X.e), X.m.stride(0), nb, R, K, R * K, K, 1, _ptr(bidx),
              _ptr(out), _ptr(oe), out.stride(0), int(kmajor), _stream(X.device))
    return out.reshape((X.L, nb) + ((K, R) if kmajor else (R, K))), oe


def align_cols(X):
    """X: MPF (..., K, N): columns aligned: (m (L, nb, K, N), column exponents (nb, N))"""
    _check(X)
    X = X.contiguous()
    K, N = X.shape[-2:]
    nb = prod(X.shape[:-2])
    out = torch.empty((X.L, nb * K * N), dtype=torch.int32, device=X.device)
    oe = torch.empty((nb, N), dtype=torch.int64, device=X.device)
    _lib.call("b3d_align", X.L, _ptr(X.m), _ptr(X.e), X.m.stride(0), nb, N, K, K * N, 1, N, None,
              _ptr(out), _ptr(oe), out.stride(0), 1, _stream(X.device))
    return out.reshape(X.L, nb, K, N), oe


def gemm_aligned(Aal, Bal):
    """(row-aligned A (L, nb, M, K), (nb, M)) x (column-aligned B (L, nb, K, N), (nb, N)) -> MPF (nb, M, N)"""
    am, ae = Aal
    bm, be = Bal
    L, nb, M, K = am.shape
    N = bm.shape[-1]
    if bm.shape[1] != nb or bm.shape[2] != K:
        raise ValueError(f"gemm shapes {tuple(am.shape)} x {tuple(bm.shape)}")
    cm = torch.empty((L, nb * M * N), dtype=torch.int32, device=am.device)
    ce = torch.empty((nb, M, N), dtype=torch.int64, device=am.device)
    _lib.call("b3d_gemm_aligned", L, _ptr(am), _ptr(ae.contiguous()), am.stride(0), _ptr(bm),
              _ptr(be.contiguous()), bm.stride(0), nb, M, N, K, _ptr(cm), _ptr(ce), cm.stride(0),
              _stream(am.device))
    return MPF(cm.reshape(L, nb, M, N), ce)


# GEMM backend: "auto" (tensor-core RNS GEMM for RNS_MIN_K <= K <= 256, the CUDA-core schoolbook GEMM otherwise),
# "rns" or "schoolbook" (both give the same bits: exact dot products, one rounding).  The threshold is measured:
# at K = 16..31 the residue GEMM is as fast as or faster than the schoolbook one on the derivative and output
# GEMMs of the bench configurations, at K = 8 it is slower.
GEMM_BACKEND = "auto"
RNS_MIN_K = 16


def _use_rns(K, M=0, N=0):
    """the residue GEMM pays for its digit split and CRT once K is large enough"""
    if GEMM_BACKEND == "schoolbook" or K > 256:
        return False
    return GEMM_BACKEND == "rns" or K >= RNS_MIN_K


def gemm(A, B, aidx=None, cache=None, key=None):
    """multiprecision (batched) product with the semantics of the reference's mpf.gemm (A aligned per row,
    B per column, exact products, one rounding per entry; reference ``recursion_gpu.py:53-79``).
    A: (M, K), (nb, M, K), or a table gathered by aidx (nb); B: (K, N) or (nb, K, N).
    cache / key: for a constant A (the caller's promise), its row-aligned form is kept in cache[(key, nb)]
    and reused by later calls."""
    batched = len(B.shape) == 3
    Bb = B if batched else B.reshape(1, *B.shape)
    nb = Bb.shape[0]
    ck = (key, nb) if cache is not None and key is not None else None
    if A is None and (ck is None or ck not in cache):
        raise ValueError("gemm: A is None and not cached")
    _check(*((A, B) if A is not None else (B,)))
    Aal = cache.get(ck) if ck is not None else None
    if Aal is not None:
        pass
    elif aidx is not None:
        Aal = align_rows(A, bidx=aidx)
    elif len(A.shape) == 2:
        Aal = align_rows(A.reshape(1, *A.shape))
        if nb > 1:
            Aal = (Aal[0].expand(-1, nb, -1, -1).contiguous(), Aal[1].expand(nb, -1).contiguous())
    else:
        Aal = align_rows(A)
    if ck is not None and ck not in cache:
        cache[ck] = Aal
    Bal = align_cols(Bb)
    C = _product(Aal, Bal)
    return C if batched else C.reshape(*C.shape[1:])


# Autotuner of the product path (opt-in): for every GEMM shape (L, batch, M, N, K) met outside stream capture,
# the candidates (schoolbook on the CUDA cores; residue GEMM with A's or B's rows on the TMEM lanes) are timed
# with CUDA events on the calling stream and the fastest is kept unless the K rule's path is within 10 %.
# Every candidate gives the same bits, so the choice only affects speed.  The schoolbook kernel skips zero
# operands, so its time depends on the data: tune on representative inputs (a CUDA-graph warm-up on zeroed
# static inputs would pick it everywhere).  Off by default: on the bench workloads the K rule is within 1 %
# of the tuned choice (cfg2 138.0 vs 137.5 ms, cfg5 377.9 vs 374.4 ms per launched step).
AUTOTUNE = False
_TUNED = {}


def _run_path(path, Aal, Bal):
    """path: "schoolbook", "rns" (the operand with more rows on the lanes), "rns_a" or "rns_b" """
    if path == "schoolbook":
        return gemm_aligned(Aal, Bal)
    from .rns import gemm_aligned_rns
    return gemm_aligned_rns(Aal, Bal, lanes={"rns_a": "a", "rns_b": "b"}.get(path))


def _candidates(K):
    out = ["schoolbook"] if K <= 64 else []
    if 8 <= K <= 256:
        out += ["rns_a", "rns_b"]
    return out or ["schoolbook"]


def _product(Aal, Bal):
    L, nb, M, K = Aal[0].shape
    N = Bal[0].shape[-1]
    if GEMM_BACKEND != "auto":
        return _run_path("rns" if _use_rns(K, M, N) else "schoolbook", Aal, Bal)
    dev = Aal[0].device
    key = (L, nb, M, N, K, dev.index)
    path = _TUNED.get(key)
    if path is None and AUTOTUNE and not torch.cuda.is_current_stream_capturing():
        default = "rns" if _use_rns(K, M, N) else "schoolbook"
        times, C = {}, None
        for cand in _candidates(K):
            _run_path(cand, Aal, Bal)                                  # warm (tables, attributes, buffers)
            best = None
            for _ in range(3):
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record()
                C = _run_path(cand, Aal, Bal)
                s1.record()
                s1.synchronize()
                best = s0.elapsed_time(s1) if best is None else min(best, s0.elapsed_time(s1))
            times[cand] = best
        fastest = min(times, key=times.get)
        ref = times.get(default) or times.get({"rns": "rns_a" if M >= N else "rns_b"}.get(default, default))
        # keep the K rule unless another path is clearly faster (timing noise must not flip a good default)
        _TUNED[key] = fastest if ref is None or times[fastest] < 0.9 * ref else default
        return C
    if path is None:
        path = "rns" if _use_rns(K, M, N) else "schoolbook"
    return _run_path(path, Aal, Bal)


def tuned_paths():
    """the autotuner's choices so far: {(L, batch, M, N, K, device): path}"""
    return dict(_TUNED)


def _elementwise(name, A, B, aidx=None, bidx=None, shape=None):
    _check(A, B)
    A, B = A.contiguous(), B.contiguous()
    if shape is None:
        shape = A.shape if aidx is None else tuple(aidx.shape)
    n = prod(shape)
    L = A.L
    cm = torch.empty((L, n), dtype=torch.int32, device=A.device)
    ce = torch.empty(n, dtype=torch.int64, device=A.device)
    ai = None if aidx is None else aidx.reshape(-1).to(device=A.device, dtype=torch.int64).contiguous()
    bi = None if bidx is None else bidx.reshape(-1).to(device=A.device, dtype=torch.int64).contiguous()
    _lib.call(name, L, _ptr(A.m), _ptr(A.e), A.m.stride(0), _ptr(ai), _ptr(B.m), _ptr(B.e), B.m.stride(0),
              _ptr(bi), n, _ptr(cm), _ptr(ce), cm.stride(0), _stream(A.device))
    return MPF(cm.reshape((L,) + tuple(shape)), ce.reshape(shape))


def mul(A, B, aidx=None, bidx=None, shape=None):
    """elementwise A * B (exact product, one rounding); optional gathers of flattened A / B"""
    return _elementwise("b3d_mul", A, B, aidx, bidx, shape)


def add(A, B, aidx=None, bidx=None, shape=None):
    """elementwise A + B (one rounding); optional gathers of flattened A / B"""
    return _elementwise("b3d_add", A, B, aidx, bidx, shape)


def random_mpf(shape, L, spread=8, device=None, generator=None):
    """random normalised values with |x| in about [2^-spread, 2^spread] (timing runs and tests; the cost
    of the path does not depend on the values; reference ``recursion_gpu.py:82-88``)"""
    n = prod(shape)
    NB = nbits(L)
    g = generator or torch.Generator().manual_seed(0)
    raw = torch.randint(-2 ** 31, 2 ** 31 - 1, (L, n), dtype=torch.int32, generator=g)
    top = NB - 32 * (L - 1)                    # bits used in the top limb
    hi = raw[L - 1].to(torch.int64) & ((1 << (top - 1)) - 1) | (1 << (top - 1))
    neg = torch.randint(0, 2, (n,), generator=g).bool()
    raw[L - 1] = hi.to(torch.int32)
    # two's complement negation of the selected columns
    m = raw.numpy().T.copy().view(np.uint32).astype(np.uint64)
    negm = neg.numpy()
    if negm.any():
        x = m[negm]
        x = (~x) & 0xFFFFFFFF
        carry = np.ones(x.shape[0], dtype=np.uint64)
        for k in range(L):
            v = x[:, k] + carry
            x[:, k] = v & 0xFFFFFFFF
            carry = v >> 32
        m[negm] = x
    mm = torch.from_numpy(m.astype(np.uint32).view(np.int32).T.copy()).reshape((L,) + tuple(shape))
    e = torch.randint(-spread, spread + 1, (n,), generator=g).reshape(shape) - NB
    return MPF(mm.to(device), e.to(device))
