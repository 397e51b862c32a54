"""blocks_3d's write_output for the xt and xt_radial coordinates on one B200: the composite linear map from
numerator coefficients (per lambda order n and log-r derivative e) to xt / xt_radial derivatives, built once
per (coordinate, Lambda, parity, Delta_1+2) in mpmath and applied to every spin, parity, structure,
coefficient and task as one multiprecision GEMM.  Host half of the reference's ``output.Output`` and
``apply_per_order`` (``blocksvibe/output.py:102-212``), same constructor and ``apply`` contract.

blocks_3d's chain (src/write_output), for one polynomial coefficient, order O = Lambda, sigma = (-1)^p:
  lambda_lr_to_lrho_lrhob  F(i, j) = 2^-(i+j) sum_{k<=i, l<=j} (-1)^(j-l) C(i,k) C(j,l) num[n = i+j-k-l][e = k+l]
                           on the triangle i + j <= O, F(j, i) = sigma F(i, j);
  congruence transforms    Z = M F M^T, M = P(Delta_1+2 / 2) R_z S (Stirling, rho -> z, power prefactor);
                           all lower triangular, so truncation to the triangle never drops a term;
  zzb_to_xt                xt(n, m) = ((m-p)/2)! / m! sum_{k<=n, l<=m} (-1)^l C(n,k) C(m,l) Z(n+m-k-l, k+l);
  lrho_to_xt_radial        xt_radial(i) = sum_j T(i, j) num[n = p][j], T = prefactor R_z S (O = Lambda - p).
An input (n, e) only feeds the antidiagonal i + j = n + e of F, which keeps the map construction O(O^4).
"""
import math

import mpmath as mp
import numpy as np
import torch

from . import mpf
from .mpf import MPF


def _rising(x, n):
    r = mp.mpf(1)
    for q in range(n):
        r *= x + q
    return r


def falling_power(x, n):
    """x (x-1) ... (x-n+1); for n < 0, 1 / ((x+1) (x+2) ... (x-n))"""
    return 1 / _rising(x + 1, -n) if n < 0 else _rising(x - n + 1, n)


def binomial(k, j):
    """C(k, j) for integer j and any integer k (negative k: the generalised coefficient), 0 for j < 0"""
    if j < 0:
        return mp.mpf(0)
    num = 1
    for q in range(j):
        num *= k - q
    return mp.mpf(num) / math.factorial(j)


def stirling_matrix(O):
    """S[n][k] = s(n, k) r_c^-n, s the signed Stirling numbers of the first kind"""
    s = [[0] * (O + 1) for _ in range(O + 1)]
    s[0][0] = 1
    for n in range(O):
        for k in range(n + 1):
            s[n + 1][k + 1] += s[n][k]
            s[n + 1][k] -= n * s[n][k]
    rc = 3 - 2 * mp.sqrt(2)
    M = mp.matrix(O + 1, O + 1)
    inv = mp.mpf(1)
    for n in range(O + 1):
        for k in range(n + 1):
            M[n, k] = s[n][k] * inv
        inv /= rc
    return M


def rho_to_z_matrix(O):
    """inverse of the z -> rho derivative map: Z[p][n] = p!/n! sum_k C(n,k) 2^-n (-1)^k (4 sqrt 2)^(n-k)
    C(-2n, p-k-n) (4 - 2 sqrt 2)^(k-n-p)"""
    r2 = mp.sqrt(2)
    a, b = 4 * r2, 4 - 2 * r2
    Z = mp.matrix(O + 1, O + 1)
    for p in range(O + 1):
        for n in range(p + 1):
            acc = mp.mpf(0)
            for k in range(n + 1):
                j = p - k - n
                if j < 0:
                    continue
                acc += binomial(n, k) * (-1) ** k * a ** (n - k) * binomial(-2 * n, j) * b ** (k - n - p)
            Z[p, n] = acc / mp.mpf(2) ** n * mp.factorial(p) / mp.factorial(n)
    return mp.inverse(Z)


def prefactor_matrix(O, D):
    """P[n][k] = falling(-D, n-k) 2^(n-k+D) C(n, k)"""
    P = mp.matrix(O + 1, O + 1)
    for n in range(O + 1):
        for k in range(n + 1):
            P[n, k] = falling_power(-D, n - k) * mp.mpf(2) ** (n - k + D) * binomial(n, k)
    return P


def one_minus_prefactor_matrix(O):
    """P[n][k] = (-1)^(n-k) falling(-1/2, n-k) 2^(n-k+1/2) C(n, k)"""
    h = mp.mpf(1) / 2
    P = mp.matrix(O + 1, O + 1)
    for n in range(O + 1):
        for k in range(n + 1):
            P[n, k] = (-1) ** (n - k) * falling_power(-h, n - k) * mp.mpf(2) ** (n - k + h) * binomial(n, k)
    return P


def binomial_products(N):
    """P[a][b] = integer coefficients (lowest degree first) of (1 + t)^a (t - 1)^b, for a + b <= N"""
    P = [[None] * (N + 1) for _ in range(N + 1)]
    P[0][0] = [1]
    for a in range(N + 1):
        for b in range(N + 1 - a):
            if a == b == 0:
                continue
            if b:
                q = P[a][b - 1]                                 # times (t - 1)
                P[a][b] = [(q[k - 1] if k else 0) - (q[k] if k < len(q) else 0) for k in range(len(q) + 1)]
            else:
                q = P[a - 1][0]                                 # times (1 + t)
                P[a][0] = [(q[k - 1] if k else 0) + (q[k] if k < len(q) else 0) for k in range(len(q) + 1)]
    return P


def xt_map(O, p, D):
    """(W (outputs x inputs) object array of mpf, inputs [(idx, e)], outputs [(n, b)]) for xt, built by pulling
    each output back through the chain (the adjoint of the step-by-step transforms).

    With the full (both-triangle) matrices, Z = M F M^T, M = P(D/2) R_z S, and Z(j, i) = sigma Z(i, j):
      output (n, b), m = p + 2 b, t = n + m:  xt = b!/m! sum_j c_j Z(t - j, j),  c_j = [u^j] (1 + u)^n (1 - u)^m
      so xt = b!/m! sum_{a, c} Y(a, c) F(a, c)  with  Y(a, c) = sum_j c_j M[t - j][a] M[j][c];
      input (idx, e), n' = p + 2 idx, s = n' + e, feeds only the antidiagonal a + c = s of F:
      F(a, s - a) = 2^-s [t^e] (1 + t)^a (t - 1)^(s - a) for a >= s - a, sigma F(s - a, a) below it.
    Every matrix is lower triangular, so no term crosses the truncation i + j <= O."""
    sigma = -1 if p % 2 else 1
    M = rho_to_z_matrix(O) * stirling_matrix(O)
    if D != 0:
        M = prefactor_matrix(O, D / 2) * M
    Mv = np.array([[M[i, k] for k in range(O + 1)] for i in range(O + 1)], dtype=object)
    inputs = [(idx, e) for idx in range((O - p) // 2 + 1) for e in range(O - (p + 2 * idx) + 1)]
    outputs = [(n, b) for n in range(O - p + 1) for b in range((O - n - p) // 2 + 1)]
    P = binomial_products(O)
    # per antidiagonal s: the inputs feeding it and F(a, s - a) per input (rows a = 0..s)
    feed = {}
    for u, (idx, e) in enumerate(inputs):
        s = p + 2 * idx + e
        col = []
        for a in range(s + 1):
            hi, lo = max(a, s - a), min(a, s - a)
            c = P[hi][lo]
            v = mp.ldexp(c[e], -s) if e < len(c) else mp.mpf(0)
            col.append(v if a >= s - a else sigma * v)
        feed.setdefault(s, ([], []))
        feed[s][0].append(u)
        feed[s][1].append(col)
    feed = {s: (us, np.array(cols, dtype=object).T) for s, (us, cols) in feed.items()}
    W = np.empty((len(outputs), len(inputs)), dtype=object)
    W[:] = mp.mpf(0)
    for o, (n, b) in enumerate(outputs):
        m = p + 2 * b
        t = n + m
        cj = P[n][m] if m % 2 == 0 else [-x for x in P[n][m]]        # (1 + u)^n (1 - u)^m
        Y = np.empty((t + 1, t + 1), dtype=object)
        Y[:] = mp.mpf(0)
        for j in range(t + 1):
            if j < len(cj) and cj[j]:
                Y[:t - j + 1, :j + 1] += cj[j] * np.outer(Mv[t - j, :t - j + 1], Mv[j, :j + 1])
        fac = mp.factorial(b) / mp.factorial(m)
        for s, (us, F) in feed.items():
            if s > t:
                continue
            anti = np.array([Y[a, s - a] for a in range(s + 1)], dtype=object)
            W[o, us] = fac * anti.dot(F)
    return W, inputs, outputs


def xt_radial_map(O, p, D):
    pre = prefactor_matrix(O, D) if p == 0 else one_minus_prefactor_matrix(O) * prefactor_matrix(O, D + 1)
    T = pre * rho_to_z_matrix(O) * stirling_matrix(O)
    W = np.empty((O + 1, O + 1), dtype=object)
    for i in range(O + 1):
        for j in range(O + 1):
            W[i, j] = T[i, j]
    return W, [(0, e) for e in range(O + 1)], [(i, 0) for i in range(O + 1)]


class Output:
    """write_output for one coordinate ("xt" | "xt_radial"), Lambda, parity (= (1 - four_pt_sign) / 2) and
    Delta_1+2 (decimal string).  Inputs: numerators of the lambda orders n = parity, parity + 2, ... <= Lambda
    (xt) or n = parity only (xt_radial), derivatives e <= Lambda - n."""

    def __init__(self, coordinate, Lam, parity, delta_1_plus_2, L, device="cuda"):
        self.coord, self.Lam, self.parity, self.L = coordinate, Lam, parity, L
        with mp.workprec(32 * L + 128):
            D = mp.mpf(delta_1_plus_2)
            if coordinate == "xt_radial":
                W, self.inputs, self.outputs = xt_radial_map(Lam - parity, parity, D)
            elif coordinate == "xt":
                W, self.inputs, self.outputs = xt_map(Lam, parity, D)
            else:
                raise ValueError(f"coordinate {coordinate!r}: only xt and xt_radial")
        self.nL = (Lam - parity) // 2 + 1
        self._idx = {}                     # cached index tensors (no host copies while a CUDA graph is captured)
        self._acache = {}                  # the row-aligned map W per batch size
        self.Wmp = W
        self.W = mpf.from_mp(list(W.reshape(-1)), L, W.shape, device)

    def apply(self, num, nL=None):
        """num: MPF (Jo, Dout, R + 1, 2, S2, nq * nL), rhs = task major, lambda-order index minor.
        Returns MPF (Jo, 2, S2, nq, outputs, Dout)."""
        Jo, Dout, R1, _, S2, B = num.shape
        nL = nL or self.nL
        nq = B // nL
        X = num.reshape(Jo, Dout, R1, 2, S2, nq, nL).permute(2, 6, 0, 3, 4, 5, 1).contiguous()   # (e, idx, ...)
        key = ("u", nL)
        if key not in self._idx:
            self._idx[key] = torch.tensor([e * nL + i for i, e in self.inputs], device=num.device)
        uidx = self._idx[key]
        X = X.reshape(R1 * nL, -1).take(uidx)
        out = mpf.gemm(self.W, X, cache=self._acache, key="W").reshape(len(self.outputs), Jo, 2, S2, nq, Dout)
        return out.permute(1, 2, 3, 4, 0, 5).contiguous()


def apply_per_order(out, nums):
    """Output.apply for numerators given per lambda order: nums[idx] MPF (Jo, Dout_n, R_n + 1, 2, S2, nq)
    (all lambda orders of the task for xt, the first for xt_radial).  Returns MPF
    (Jo, 2, S2, nq, outputs, max Dout) (reference ``output.py:193-212``)."""
    Dmax = max(x.shape[1] for x in nums)
    rows = []
    for idx, x in enumerate(nums):
        need = [e for i, e in out.inputs if i == idx]
        if not need:
            continue
        Jo, D, R1, _, S2, nq = x.shape
        X = x.permute(2, 0, 3, 4, 5, 1).contiguous()                                             # (e, jo, p, s, q, d)
        if D < Dmax:
            X = mpf.cat([X, mpf.zeros((R1, Jo, 2, S2, nq, Dmax - D), x.L, x.device)], 5)
        key = ("need", idx)
        if key not in out._idx:
            out._idx[key] = torch.tensor(need, device=x.device)
        rows.append(X.reshape(R1, -1).take(out._idx[key]))
    X = mpf.cat(rows, 0)
    Jo, _, _, _, S2, nq = nums[0].shape
    res = mpf.gemm(out.W, X, cache=out._acache, key="W").reshape(len(out.outputs), Jo, 2, S2, nq, Dmax)
    return res.permute(1, 2, 3, 4, 0, 5).contiguous()
