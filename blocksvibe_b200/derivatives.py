"""blocks_3d's post-recursion stages on one B200: residues -> log(r) derivatives at r_c -> r^Delta restored
-> Delta -> x shift -> numerator polynomials (with pole shifting), for every internal spin, parity,
structure and right-hand side of a batched recursion.  Host half of the reference's ``derivatives.Derivs``
(``blocksvibe/derivatives.py:313-582``): same constructor, ``for_order``, ``start``, ``accumulate``,
``finish`` / ``finish_iter`` contract.

Per (spin j, parity, structure), with w[k][n] = n^k r_c^n (r_c = 3 - 2 sqrt 2), R = Lambda - n_lambda,
poles i of spin j at full order (positions D_i = d_i / 2, shifts s_i), x = Delta - ub_j (blocks_3d's
conformal_block_derivatives, restore_r_delta, shift_block, together_with_factors):

  c[k]    = sum_m w[k][m] h_inf[m]                         v_i[k] = sum_m w[k][m + s_i] res[m][i]
  a_i[e]  = sum_{d <= e} C(e, d) D_i^(e-d) v_i[d]          G[d][w] = sum_i D_i^w v_i[d]
  P_e[t]  = C(e, t) c[e-t] + sum_{u=t+1}^{e} C(e, u) G[e-u][u-t-1]
  num_e(x) = P_e(x + ub) Pi(x) + sum_i a_i[e] Pi_i(x),   Pi = prod_i (x - x_i),  Pi_i = Pi / (x - x_i)

The moments v are accumulated during the recursion (one kernel per level, libb3dgpu b3d_moments_level);
c, a, G, the polynomial part and the numerators are multiprecision GEMMs.  The numerator matrix
A_j = [Pi_i(x) | Pi(x) (x + ub)^t] is exact: in y = 2x the roots are integers.  Pole shifting
(kept_pole_order < order) replaces the unprotected poles by the kept ones with residues S a,
S = A^-1 V (blocks_3d's shift_poles); its closed form S_ki = (y'_k / y_i)^h l_k(y_i) (l_k the Lagrange
basis on the kept poles y', h = #kept // 2) is exact in rationals and folded into the numerator matrix.
"""
from fractions import Fraction
from math import comb, lcm

import mpmath as mp
import numpy as np
import torch

from . import _lib, mpf, structure as S
from .mpf import MPF


# ---------------------------------------------------------------- exact integer polynomial helpers

def poly_times_linear(p, a):
    """p(y) (y + a), integer coefficients lowest first"""
    out = [0] * (len(p) + 1)
    for k, c in enumerate(p):
        out[k] += a * c
        out[k + 1] += c
    return out


def divide_by_roots(p, roots):
    """[p(y) / (y - r) for r in roots], each r a root of p (exact synthetic division)"""
    n = len(p) - 1
    out = []
    for r in roots:
        q, acc = [0] * n, 0
        for k in range(n, 0, -1):
            acc = p[k] + r * acc
            q[k - 1] = acc
        if p[0] + r * acc != 0:
            raise ValueError("not a root")
        out.append(q)
    return out


def shifted_pole_columns(roots, new, comp):
    """Numerator columns of blocks_3d's pole shifting, exact.  roots: old poles y_i = 2 x_i; new: the
    protected old poles (y = 0) then the kept poles y'_k; comp[q] = Pi_new(y) / (y - new[q]).
    Returns per old pole (polynomial numerator coefficients, positive integer denominator):
    protected pole -> comp of its slot; unprotected pole i -> sum_k S_ki comp[nprot + k] with
    S_ki = (y'_k / y_i)^h prod_{m != k} (y_i - y'_m) / (y'_k - y'_m), h = #kept // 2."""
    nprot = sum(1 for y in new if y == 0)
    keep = new[nprot:]
    size = len(keep)
    h = size // 2
    dk = []
    for k in range(size):
        d = 1
        for mm in range(size):
            if mm != k:
                d *= keep[k] - keep[mm]
        dk.append(d)
    common = 1
    for d in dk:
        common = lcm(common, abs(d))
    weight = [keep[k] ** h * (common // abs(dk[k])) * (1 if dk[k] > 0 else -1) for k in range(size)]
    ncoef = len(comp[0]) if comp else 1
    cols = []
    for y in roots:
        if y == 0:
            cols.append((list(comp[new.index(0)]), 1))
            continue
        if size == 0:
            cols.append(([0] * ncoef, 1))
            continue
        poly = [0] * ncoef
        for k in range(size):
            f = weight[k]
            for mm in range(size):
                if mm != k:
                    f *= y - keep[mm]
            if f:
                for c, v in enumerate(comp[nprot + k]):
                    poly[c] += f * v
        den = y ** h * common
        if den < 0:
            den, poly = -den, [-v for v in poly]
        cols.append((poly, den))
    return cols


def _take_rows(X, idx):
    return X.take(idx)


class Derivs:
    """Post-recursion stages for one Plan and any batch of right-hand sides with lambda orders
    n >= Lambda - R.  two_js: internal spins to output (default: all two_j <= two_j_max)."""

    def __init__(self, plan, R, L, two_js=None, kept_pole_order=None, device="cuda"):
        self.plan, self.R, self.L, self.device = plan, R, L, torch.device(device)
        order = plan.order
        self.kept = kept_pole_order if kept_pole_order is not None and kept_pole_order < order else None
        tj12, tj43, tjmax = plan.tj12, plan.tj43, plan.tjmax
        self.tjs = list(two_js) if two_js is not None else list(range(tj12 % 2, tjmax + 1, 2))
        self.Jo = Jo = len(self.tjs)
        self.poles = [S.block_poles(tj, tj12, tj43, order) for tj in self.tjs]
        self.NP = NP = max(len(p) for p in self.poles)
        self.NPout = NP if self.kept is None else max(len(S.block_poles(tj, tj12, tj43, self.kept)) for tj in self.tjs)
        self.Dout = self.NPout + R + 1
        self._moment_levels()
        self._constants()
        # index tensors of finish_iter, built once (no host-to-device copies while a CUDA graph is captured)
        self._jidx = torch.tensor([(tj - tj12 % 2) // 2 for tj in self.tjs], device=self.device)
        self._orders = {}
        self._acache = {}                  # row-aligned constant GEMM operands (shared by the for_order copies)

    # ------------------------------------------------------------ moment bookkeeping per level
    def _moment_levels(self):
        pl, order, Jo, NP = self.plan, self.plan.order, self.Jo, self.NP
        tjo = np.array(self.tjs, dtype=np.int64)
        pos = {tj: jo for jo, tj in enumerate(self.tjs)}
        self.levels = []
        for m in range(order):
            tjs = pl._tjs[m]
            sel = np.flatnonzero(np.isin(tjs, tjo))
            npol = pl._npol[m][sel]
            tot = int(npol.sum())
            if tot == 0:
                self.levels.append(None)
                continue
            rep = np.repeat(np.arange(len(sel)), npol)
            pidx = np.arange(tot) - np.repeat(np.cumsum(npol) - npol, npol)
            jidx = sel[rep]
            tj = tjs[jidx]
            jo = np.array([pos[int(x)] for x in tj], dtype=np.int64)
            kind, k = S.pole_at_v(tj, pl.tj12, pl.tj43, pl._ords[m][jidx], pidx)
            i = S.pole_index_v(tj, pl.tj12, pl.tj43, order, kind, k)
            nn = m + S.level_shift_v(kind, k)
            jidx, pidx, jo, i, nn = (np.repeat(a, 2) for a in (jidx, pidx, jo, i, nn))
            p = np.tile(np.array([0, 1], dtype=np.int64), tot)
            ph = pl.phys_slots(p * pl.nslots + pl._flat[pl._start[m] + jidx] + pidx)
            ok = ph != pl.zero_slot
            if not ok.any():
                self.levels.append(None)
                continue
            dev = self.device
            self.levels.append((torch.as_tensor(ph[ok], device=dev), torch.as_tensor(((p * Jo + jo) * NP + i)[ok], device=dev),
                                torch.as_tensor(nn[ok].astype(np.int64), device=dev)))

    # ------------------------------------------------------------ constants (once per operator and R)
    def _constants(self):
        L, R, order, Jo, NP, dev = self.L, self.R, self.plan.order, self.Jo, self.NP, self.device
        with mp.workprec(32 * L + 64):
            rc = 3 - 2 * mp.sqrt(2)
            pw = [rc ** n for n in range(order + 1)]
            self.rcpow = mpf.from_mp(pw, L, (order + 1,), dev)
            self.Wh = mpf.from_mp([(mp.mpf(n) ** k if (n or k) else 1) * pw[n] for k in range(R + 1) for n in range(order + 1)],
                                  L, (R + 1, order + 1), dev)
        # C(e, k) D^(e-k) = C(e, k) d^(e-k) 2^(k-e) per distinct d = 2 D (index 0: zeros)
        d2 = sorted({S.twice_position(P, tj) for tj, pl in zip(self.tjs, self.poles) for P in pl})
        di = {d: q + 1 for q, d in enumerate(d2)}
        ints, exps = [0] * (R + 1) ** 2, [0] * (R + 1) ** 2
        for d in d2:
            for e in range(R + 1):
                ints += [comb(e, k) * d ** (e - k) if k <= e else 0 for k in range(R + 1)]
                exps += [k - e for k in range(R + 1)]
        self.Ttab = mpf.from_ints(ints, exps, L, (len(d2) + 1, R + 1, R + 1), dev)
        didx = np.zeros((Jo, NP), dtype=np.int64)
        for jo, (tj, pl) in enumerate(zip(self.tjs, self.poles)):
            didx[jo, :len(pl)] = [di[S.twice_position(P, tj)] for P in pl]
        self.didx = torch.as_tensor(didx, device=dev)
        self._small_constants()
        self.Anum = self._numerator_matrix()

    def _numerator_matrix(self):
        """A_j (Jo, Dout, NP + R + 1): columns Pi_i(x) (or the pole-shifted combinations), then
        Pi(x) (x + ub)^t for t <= R; exact integers in y = 2x, rounded once"""
        L, R, NP, Jo, Dout = self.L, self.R, self.NP, self.Jo, self.Dout
        W = NP + R + 1
        tj12, tj43 = self.plan.tj12, self.plan.tj43
        vals = [Fraction(0)] * (Jo * Dout * W)
        for jo, (tj, pl) in enumerate(zip(self.tjs, self.poles)):
            two_ub = tj + 1 if tj <= 1 else tj + 2
            roots = [S.twice_position(P, tj) - two_ub for P in pl]
            if self.kept is None:
                new = roots
            else:
                new = [y for y in roots if y == 0] + [S.twice_position(P, tj) - two_ub
                                                      for P in S.block_poles(tj, tj12, tj43, self.kept)
                                                      if S.twice_position(P, tj) != two_ub]
            npj = len(new)
            if npj + R + 1 > Dout:
                raise ValueError(f"spin {tj}: {npj} poles after shifting exceed the output width")
            Pi = [1]
            for y0 in new:
                Pi = poly_times_linear(Pi, -y0)
            cols = []                                             # (column, integer poly, scale, denominator)
            q = Pi
            for t in range(R + 1):
                cols.append((NP + t, q, npj + t, 1))
                q = poly_times_linear(q, two_ub)
            comp = divide_by_roots(Pi, new) if new else []
            if self.kept is None:
                cols += [(i, c, npj - 1, 1) for i, c in enumerate(comp)]
            else:
                cols += [(i, poly, npj - 1, den) for i, (poly, den) in enumerate(shifted_pole_columns(roots, new, comp))]
            for col, poly, sc, den in cols:                       # x^k coefficient = poly[k] / den 2^(k - sc)
                for k, v in enumerate(poly):
                    if v:
                        vals[(jo * Dout + k) * W + col] = Fraction(v, den) * Fraction(2) ** (k - sc)
        return mpf.from_fractions(vals, L, (Jo, Dout, W), self.device)

    def _small_constants(self):
        """R-dependent tables of the polynomial part: H[e][s] = sum_d C(e, d) G'[s][d] with
        G'[s][d] = G[s - 1 - d][d], P_e[t] = C(e, t) c[e - t] + H[e][e - t]"""
        L, R, dev = self.L, self.R, self.device
        R1 = R + 1
        self.Cb = mpf.from_ints([comb(e, d) for e in range(R1) for d in range(R1)], [0] * R1 * R1, L, (R1, R1), dev)
        Rw = max(R, 1)
        self.gidx = torch.tensor([(s - 1 - d) * R1 + d if 1 <= s and d <= s - 1 else Rw * R1
                                  for s in range(R1) for d in range(R1)], device=dev)
        te = [(t, e) for t in range(R1) for e in range(R1)]
        self.cidx_te = torch.tensor([e - t if t <= e else R1 for t, e in te], device=dev)
        self.hidx_te = torch.tensor([e * R1 + (e - t) if t <= e else R1 * R1 for t, e in te], device=dev)
        self.cb_te = mpf.from_ints([comb(e, t) if t <= e else 0 for t, e in te], [0] * len(te), L, (len(te),), dev)
        self._cb_rows = {}

    def for_order(self, R):
        """the same stages for a smaller R (a higher lambda order of the task), sharing this object's
        constants as slices (reference ``derivatives.py:434-446``).  The constants of each R are built once;
        every call returns a fresh object (its accumulators are its own)."""
        if R > self.R:
            raise ValueError(f"R = {R} > {self.R}")
        base = self._orders.get(R)
        if base is None:
            base = object.__new__(Derivs)
            base.__dict__.update(self.__dict__)
            base.R, base.Dout = R, self.NPout + R + 1
            R1, K = R + 1, self.NP + R + 1
            base.Anum = MPF(self.Anum.m[:, :, :base.Dout, :K], self.Anum.e[:, :base.Dout, :K]).contiguous()
            base.Ttab = MPF(self.Ttab.m[:, :, :R1, :R1], self.Ttab.e[:, :R1, :R1]).contiguous()
            base.Wh = MPF(self.Wh.m[:, :R1], self.Wh.e[:R1]).contiguous()
            base._small_constants()
            base._orders = {}
            self._orders[R] = base
        d = object.__new__(Derivs)
        d.__dict__.update(base.__dict__)
        return d

    def footprint_bytes(self, B):
        """device bytes of the moment accumulators for B right-hand sides"""
        return (4 * self.L + 8) * 2 * self.Jo * self.NP * (self.R + 1) * self.plan.Smax ** 2 * B

    # ------------------------------------------------------------ accumulation during the recursion
    def start(self, B):
        """zero moment accumulators (rows, R + 1, S^2 B) for a batch of B right-hand sides"""
        self.B = B
        self.N = self.plan.Smax ** 2 * B
        self.mom = mpf.zeros((2 * self.Jo * self.NP, self.R + 1, self.N), self.L, self.device)

    def accumulate(self, m, res):
        """recursion hook: add level m's residues of the output spins to the moments"""
        lev = self.levels[m]
        if lev is None:
            return
        sl, rw, nn = lev
        p = lambda t: t.data_ptr()
        _lib.call("b3d_moments_level", self.L, p(res.m), p(res.e), res.m.stride(0), p(self.rcpow.m), p(self.rcpow.e),
                  self.rcpow.m.stride(0), p(sl), p(rw), p(nn), sl.numel(), self.N, self.R + 1,
                  p(self.mom.m), p(self.mom.e), self.mom.m.stride(0), torch.cuda.current_stream(self.device).cuda_stream)

    # ------------------------------------------------------------ final GEMMs
    def finish(self, h_inf, chunk=None):
        """h_inf: MPF (2, order + 1, Jh, Smax^2, B).  Returns numerators MPF (Jo, Dout, R + 1, 2, Smax^2, B):
        [spin, x^k coefficient, log r derivative e, parity, structure a * Smax + b, rhs]"""
        return mpf.cat([num for _, num in self.finish_iter(h_inf, chunk)], 0)

    def finish_iter(self, h_inf, chunk=None):
        """as finish, by chunks of output spins: yields (first spin index, numerators)"""
        R, Jo, NP, order, L, dev = self.R, self.Jo, self.NP, self.plan.order, self.L, self.device
        R1, N, Rw = R + 1, self.N, max(R, 1)
        S2 = self.plan.Smax ** 2
        Nc = 2 * N
        jidx = self._jidx
        H = MPF(h_inf.m[:, :, :order + 1][:, :, :, jidx], h_inf.e[:, :order + 1][:, :, jidx])   # (2, o+1, Jo, S2, B)
        H = H.permute(1, 2, 0, 3, 4).contiguous().reshape(order + 1, Jo * Nc)
        ac = self._acache
        c = mpf.gemm(self.Wh, H, cache=ac, key=("Wh", R)).reshape(R1, Jo, Nc).permute(1, 0, 2)  # (Jo, R+1, Nc)
        mom = self.mom.reshape(2, Jo, NP, R1, N)
        chunk = chunk or Jo
        for j0 in range(0, Jo, chunk):
            j1 = min(Jo, j0 + chunk)
            J = j1 - j0
            v = mom[:, j0:j1].permute(1, 2, 3, 0, 4).contiguous().reshape(J, NP, R1, Nc)           # v_i[d]
            di = self.didx[j0:j1].reshape(-1)
            a = mpf.gemm(self.Ttab, v.reshape(J * NP, R1, Nc), aidx=di, cache=ac,
                         key=("Ttab", R, j0, j1)).reshape(J, NP, R1, Nc)                            # a_i[e]
            vkey = ("Vand", R, j0, j1)
            if (vkey, J) not in ac:
                T = self.Ttab.take(di).reshape(J, NP, R1, R1)                                      # [.., w, 0] = D_i^w
                Vand = MPF(T.m[:, :, :, :Rw, 0].permute(0, 1, 3, 2), T.e[:, :, :Rw, 0].permute(0, 2, 1)).contiguous()
            else:
                Vand = None
            G = mpf.gemm(Vand, v.reshape(J, NP, R1 * Nc), cache=ac, key=vkey).reshape(J, Rw * R1, Nc)  # G[w][d]
            Gz = mpf.cat([G, mpf.zeros((J, 1, Nc), L, dev)], 1)
            Gs = Gz.permute(1, 0, 2).contiguous().take(self.gidx).reshape(R1, R1, J, Nc)          # (s, d, jo, col)
            Gs = Gs.permute(1, 2, 0, 3).contiguous().reshape(R1, J * R1 * Nc)                     # (d, jo s col)
            Hm = mpf.gemm(self.Cb, Gs, cache=ac, key=("Cb", R)).reshape(R1, J, R1, Nc)           # H[e][s]
            Hm = mpf.cat([Hm.permute(0, 2, 1, 3).contiguous().reshape(R1 * R1, J, Nc),
                          mpf.zeros((1, J, Nc), L, dev)], 0)
            cz = mpf.cat([c[j0:j1].permute(1, 0, 2).contiguous(), mpf.zeros((1, J, Nc), L, dev)], 0)  # (d | 0, jo, col)
            T2 = R1 * R1
            cte = cz.take(self.cidx_te).contiguous()                                              # (T2, J, Nc)
            key = J * Nc
            if key not in self._cb_rows:
                self._cb_rows[key] = torch.arange(T2, device=dev).repeat_interleave(J * Nc)
            P = mpf.mul(cte.reshape(-1), self.cb_te, bidx=self._cb_rows[key], shape=(T2, J, Nc))
            P = mpf.add(P, Hm.take(self.hidx_te).contiguous())                                    # ((t, e), jo, col)
            P = P.reshape(R1, R1, J, Nc).permute(2, 0, 1, 3).contiguous().reshape(J, R1, R1 * Nc)  # (jo, t, e col)
            Bn = mpf.cat([a.reshape(J, NP, R1 * Nc), P], 1)                                       # (jo, i | t, e col)
            num = mpf.gemm(self.Anum[j0:j1], Bn, cache=ac, key=("Anum", R, j0, j1))               # (J, Dout, R+1 Nc)
            yield j0, num.reshape(J, self.Dout, R1, 2, S2, self.B)
