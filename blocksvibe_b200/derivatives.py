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

The moments v are accumulated during the recursion: each level's terms res r_c^n are staged
(b3d_moments_stage) and the moments of a window of levels are formed once (b3d_moments_flush; the
per-level read-modify-write form b3d_moments_level is kept as MOMENTS = "per_level"); c, a, G, the polynomial
part and the numerators are multiprecision GEMMs, at derivative_limbs(L, R, order) limbs.  The numerator matrix
A_j = [Pi_i(x) | Pi(x) (x + ub)^t] is exact: in y = 2x the roots are integers.  Pole shifting
(kept_pole_order < order) replaces the unprotected poles by the kept ones (blocks_3d's shift_poles); the
replaced pole's column has the closed form of numerator_basis_y, exact in rationals and folded into the
numerator matrix.
"""
from fractions import Fraction
from math import comb

import mpmath as mp
import numpy as np
import torch

from . import _lib, mpf, structure as S
from .mpf import MPF


def derivative_limbs(L, R, order):
    """limbs of the derivative stages for recursion limbs L: the binomial sums of the stages (a_i[e] from the
    moments, the polynomial part from D_i^w times moments) cancel terms up to about (2 order)^R larger than their
    result, so where R log2(order) + 16 bits exceed the 62 bits by which L limbs exceed the task's precision, the
    stages run with L + 4 limbs (128 more bits) and the results are rounded back to L limbs"""
    guard = R * max(1.0, float(np.log2(max(order, 2)))) + 16
    if guard <= 62 or MOMENTS != "staged":
        return L
    wide = L + 4
    if not _lib.lib().b3d_supported_limbs(wide):
        raise _lib.B3DError(f"no kernels compiled for the derivative stages' {wide} limbs")
    return wide


def resize(X, Lout):
    """X with Lout limbs (L or L +- 4): widening exact, narrowing rounded once"""
    if X.L == Lout:
        return X
    n = X.numel()
    X = X.contiguous()
    om = torch.empty((Lout,) + tuple(X.shape), dtype=torch.int32, device=X.device)
    oe = torch.empty(tuple(X.shape), dtype=torch.int64, device=X.device)
    _lib.call("b3d_resize", X.L, X.m.data_ptr(), X.e.data_ptr(), X.m.stride(0) if n else 0, n, Lout, om.data_ptr(),
              oe.data_ptr(), om.stride(0) if n else 0, torch.cuda.current_stream(X.device).cuda_stream)
    return MPF(om, oe)


# Moments: "staged" (each level stages its terms, exact window sums flushed once per window: b3d_moments_stage /
# b3d_moments_flush) or "per_level" (read-modify-write of every moment at every level: b3d_moments_level).
MOMENTS = "staged"
STAGE_BYTES = 4 << 30           # device bytes of the staging window (whole levels; at least one)


# ---------------------------------------------------------------- numerator basis (exact rationals)

def _poly_from_roots(roots):
    """prod (y - r), coefficients lowest degree first"""
    p = [Fraction(1)]
    for r in roots:
        p = [Fraction(0)] + p
        for i in range(len(p) - 1):
            p[i] -= r * p[i + 1]
    return p


def _deflate(p, r):
    """(quotient, remainder) of p(y) by (y - r) (Horner)"""
    q, acc = [Fraction(0)] * (len(p) - 1), Fraction(0)
    for i in range(len(p) - 1, 0, -1):
        acc = p[i] + r * acc
        q[i - 1] = acc
    return q, p[0] + r * acc if p else Fraction(0)


def numerator_basis_y(tj, tj12, tj43, order, kept=None, R=0):
    """The numerator basis of one spin in y = 2x (every pole position is then an integer y_i = 2 D_i - 2 ub):
    (pole columns, polynomial columns, npj).  Pole column i multiplies the residue a_i of the i-th pole of the
    spin at full order; polynomial column t = Pi(y) (y + 2 ub)^t multiplies the polynomial part; Pi is the
    product over the output poles: the protected old poles (y = 0) and the kept ones (all other old poles
    without pole shifting, else the nonzero poles of the block at kept_pole_order), npj of them.

    Column of an old pole y_i, with Pi = y^z Pk(y) (z protected poles, Pk over the kept ones, h = #kept // 2):
        y_i = 0:  Pi(y) / y
        else:     y^z (Pk(y) - (y / y_i)^h Pk(y_i)) / (y - y_i)
    Without pole shifting y_i is a root of Pk and this is Pi / (y - y_i).  With pole shifting it is blocks_3d's
    replacement of the pole (shift_poles: residues A^-1 V a on the kept poles, A[r][k] = y'_k^(r - h),
    V[r][i] = y_i^(r - h)): sum_k S_ki Pi / (y - y'_k) with S_ki = (y'_k / y_i)^h l_k(y_i), l_k the Lagrange
    basis of the kept poles, which sums to the closed form above because y^h (h < #kept) is interpolated
    exactly on the kept poles."""
    two_ub = tj + 1 if tj <= 1 else tj + 2
    ys = [S.twice_position(P, tj) - two_ub for P in S.block_poles(tj, tj12, tj43, order)]
    pool = ys if kept is None else [S.twice_position(P, tj) - two_ub for P in S.block_poles(tj, tj12, tj43, kept)]
    keep = [y for y in pool if y != 0]
    z = ys.count(0)
    h = len(keep) // 2
    Pk = _poly_from_roots(keep)
    Pi = [Fraction(0)] * z + Pk
    pole_cols = []
    for yi in ys:
        if yi == 0:
            pole_cols.append(Pi[1:])
            continue
        c = sum(v * Fraction(yi) ** k for k, v in enumerate(Pk)) / Fraction(yi) ** h
        N = list(Pk)
        N[h] -= c
        q, rem = _deflate(N, yi)
        if rem != 0:
            raise ArithmeticError("pole column is not a polynomial")
        pole_cols.append([Fraction(0)] * z + q)
    poly_cols, q = [], Pi
    for t in range(R + 1):
        poly_cols.append(q)
        q = [Fraction(0)] + q
        for i in range(len(q) - 1):
            q[i] += two_ub * q[i + 1]
    return pole_cols, poly_cols, z + len(keep)


def to_x(poly_y, scale):
    """coefficients in x of 2^-scale p(2x)"""
    return [v * Fraction(2) ** (k - scale) for k, v in enumerate(poly_y)]


# per-run attributes (set by start / accumulate / flush): never shared through the for_order constants
_RUN_STATE = ("B", "N", "mom", "_stage", "_staged_mode", "_W", "_m0", "_last", "_flushes")


class Derivs:
    """Post-recursion stages for one Plan and any batch of right-hand sides with lambda orders
    n >= Lambda - R.  two_js: internal spins to output (default: all two_j <= two_j_max)."""

    def __init__(self, plan, R, L, two_js=None, kept_pole_order=None, device="cuda", Ld=None):
        """L: limbs of the residues; Ld: limbs of the derivative stages and of the numerators they return
        (default derivative_limbs(L, R, order))"""
        self.plan, self.R, self.L, self.device = plan, R, L, torch.device(device)
        self.Ld = Ld if Ld is not None else derivative_limbs(L, R, plan.order)
        if self.Ld not in (L, L + 4) or (self.Ld != L and MOMENTS != "staged"):
            raise ValueError(f"derivative limbs {self.Ld} for residues of {L} limbs (L or L + 4, staged moments)")
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
        """per level: (slots, moment rows, n) of the pole-step tasks whose spin is an output spin: the residue
        of task (p, tj, pole) at level m feeds moment row (p Jo + jo) NP + i (i: the pole's index in the block at
        full order) with weight n^k r_c^n, n = m + shift(pole)"""
        pl, Jo, NP, dev = self.plan, self.Jo, self.NP, self.device
        shift = np.zeros((2, Jo, NP), dtype=np.int64)              # level shift of each row's pole
        for jo, poles in enumerate(self.poles):
            shift[:, jo, :len(poles)] = [S.level_shift(P) for P in poles]
        self._row_shift = torch.as_tensor(shift.reshape(-1), device=dev)
        jo_of = np.full(pl.tjmax + 2 * pl.order + 3, -1, dtype=np.int64)
        jo_of[np.array(self.tjs, dtype=np.int64)] = np.arange(Jo)
        self.levels = []
        for lev in pl.levels:
            jo = None if lev is None else jo_of[lev["t_tj"]]
            if jo is None or not (jo >= 0).any():
                self.levels.append(None)
                continue
            sel = jo >= 0
            tj, kind, k = lev["t_tj"][sel], lev["t_kind"][sel], lev["t_k"][sel]
            i = S.pole_index_v(tj, pl.tj12, pl.tj43, pl.order, kind, k)
            row = (lev["t_p"][sel] * Jo + jo[sel]) * NP + i
            n = lev["m"] + S.level_shift_v(kind, k)
            self.levels.append(tuple(torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int64, device=dev)
                                     for a in (lev["t_slot"][sel], row, n)))

    # ------------------------------------------------------------ constants (once per operator and R)
    def _constants(self):
        L, R, order, Jo, NP, dev = self.Ld, self.R, self.plan.order, self.Jo, self.NP, self.device
        with mp.workprec(32 * L + 64):
            rc = 3 - 2 * mp.sqrt(2)
            pw = [rc ** n for n in range(order + 1)]
            self.rcpow = mpf.from_mp(pw, self.L, (order + 1,), dev)       # the staged terms: residue limbs
            self.Wh = mpf.from_mp([(mp.mpf(n) ** k if (n or k) else 1) * pw[n] for k in range(R + 1) for n in range(order + 1)],
                                  L, (R + 1, order + 1), dev)
        # the shift of a polynomial in log r by a pole position D: T(D)[e][k] = C(e, k) D^(e - k), a Pascal matrix
        # (T[e][k] = T[e-1][k-1] + D T[e-1][k]); one table per distinct position, row 0 of the table all zero
        twice = [[S.twice_position(P, tj) for P in pl] for tj, pl in zip(self.tjs, self.poles)]
        positions = np.unique(np.concatenate([np.array(t, dtype=np.int64) for t in twice]))
        tables = [[Fraction(0)] * (R + 1) ** 2]
        for d in positions.tolist():
            D = Fraction(int(d), 2)
            T = [[Fraction(0)] * (R + 1) for _ in range(R + 1)]
            T[0][0] = Fraction(1)
            for e in range(1, R + 1):
                for k in range(e + 1):
                    T[e][k] = (T[e - 1][k - 1] if k else 0) + D * T[e - 1][k]
            tables.append([x for row in T for x in row])
        self.Ttab = mpf.from_fractions([x for t in tables for x in t], L, (len(tables), R + 1, R + 1), dev)
        self._power_tables()
        didx = np.zeros((Jo, NP), dtype=np.int64)
        for jo, t in enumerate(twice):
            didx[jo, :len(t)] = np.searchsorted(positions, t) + 1
        self.didx = torch.as_tensor(didx, device=dev)
        self._small_constants()
        self.Anum = self._numerator_matrix()

    def _power_tables(self):
        """n^k (k <= R, n <= order) as KW 32-bit limbs and their bit lengths, for the staged moments' flush"""
        R1, NN = self.R + 1, self.plan.order + 1
        need = max(1, -(-(max(n ** k for k in range(R1) for n in range(NN))).bit_length() // 32))
        KW = next((w for w in (2, 6, 12) if w >= need), None)
        if KW is None:
            raise ValueError(f"n^k up to {self.plan.order}^{self.R} exceeds the flush kernel's 12 limbs")
        limbs = np.zeros((R1, NN, KW), dtype=np.uint32)
        bits = np.zeros((R1, NN), dtype=np.int32)
        for k in range(R1):
            for n in range(NN):
                v = n ** k                                   # 0^0 = 1
                bits[k, n] = v.bit_length()
                for j in range(KW):
                    limbs[k, n, j] = (v >> (32 * j)) & 0xFFFFFFFF
        self._nk = torch.as_tensor(limbs.view(np.int32), device=self.device)
        self._nkb = torch.as_tensor(bits, device=self.device)
        self._KW = KW

    def _numerator_matrix(self):
        """A (Jo, Dout, NP + R + 1): per spin, the numerator basis (numerator_basis_y) in x, pole columns first
        (padded to NP), then the R + 1 polynomial columns; exact rationals rounded once"""
        R, NP, Jo, Dout = self.R, self.NP, self.Jo, self.Dout
        W = NP + R + 1
        A = np.full((Jo, Dout, W), Fraction(0), dtype=object)
        for jo, tj in enumerate(self.tjs):
            poles, polys, npj = numerator_basis_y(tj, self.plan.tj12, self.plan.tj43, self.plan.order, self.kept, R)
            if npj + R + 1 > Dout:
                raise ValueError(f"spin {tj}: {npj} poles after shifting exceed the output width")
            for i, poly in enumerate(poles):
                A[jo, :len(poly), i] = to_x(poly, npj - 1)
            for t, poly in enumerate(polys):
                A[jo, :len(poly), NP + t] = to_x(poly, npj + t)
        return mpf.from_fractions(list(A.reshape(-1)), self.Ld, (Jo, Dout, W), self.device)

    def _small_constants(self):
        """R-dependent tables of the polynomial part: H[e][s] = sum_d C(e, d) G'[s][d] with
        G'[s][d] = G[s - 1 - d][d], P_e[t] = C(e, t) c[e - t] + H[e][e - t]"""
        L, R, dev = self.Ld, self.R, self.device
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
            base.__dict__.update({k: v for k, v in self.__dict__.items() if k not in _RUN_STATE})
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

    def stage_window(self, B):
        """levels per staging window for B right-hand sides (the whole order when it fits STAGE_BYTES)"""
        per_level = (4 * self.L + 8) * 2 * self.Jo * self.NP * self.plan.Smax ** 2 * B
        return int(max(1, min(self.plan.order, STAGE_BYTES // max(per_level, 1))))

    def footprint_bytes(self, B):
        """device bytes of the moment accumulators (and the staging window) for B right-hand sides"""
        per = 2 * self.Jo * self.NP * self.plan.Smax ** 2 * B
        return per * ((4 * self.Ld + 8) * (self.R + 1) + (4 * self.L + 8) * (self.stage_window(B) if MOMENTS == "staged" else 0))

    # ------------------------------------------------------------ accumulation during the recursion
    def start(self, B):
        """zero moment accumulators (rows, R + 1, S^2 B) for a batch of B right-hand sides"""
        self.B = B
        self.N = self.plan.Smax ** 2 * B
        rows = 2 * self.Jo * self.NP
        self.mom = mpf.zeros((rows, self.R + 1, self.N), self.Ld, self.device)
        self._staged_mode = MOMENTS == "staged"
        if self._staged_mode:
            self._W = self.stage_window(B)
            self._stage = mpf.zeros((self._W, rows, self.N), self.L, self.device)
            self._m0, self._last, self._flushes = 0, None, 0

    def accumulate(self, m, res):
        """recursion hook: add level m's residues of the output spins to the moments (staged: into the window,
        flushed into the moments when the window is full)"""
        lev = self.levels[m]
        if lev is None:
            return
        sl, rw, nn = lev
        p = lambda t: t.data_ptr()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        if not self._staged_mode:
            _lib.call("b3d_moments_level", self.L, p(res.m), p(res.e), res.m.stride(0), p(self.rcpow.m), p(self.rcpow.e),
                      self.rcpow.m.stride(0), p(sl), p(rw), p(nn), sl.numel(), self.N, self.R + 1,
                      p(self.mom.m), p(self.mom.e), self.mom.m.stride(0), stream)
            return
        if m - self._m0 >= self._W:
            self.flush()
            self._m0 = m
        rows = 2 * self.Jo * self.NP
        _lib.call("b3d_moments_stage", self.L, p(res.m), p(res.e), res.m.stride(0), p(self.rcpow.m), p(self.rcpow.e),
                  self.rcpow.m.stride(0), p(sl), p(rw), p(nn), sl.numel(), self.N, m - self._m0, rows,
                  p(self._stage.m), p(self._stage.e), self._stage.m.stride(0), stream)
        self._last = m

    def flush(self):
        """form the moments of the staged window (no-op without staged levels); the window is then empty"""
        if not getattr(self, "_staged_mode", False) or self._last is None:
            return
        p = lambda t: t.data_ptr()
        rows, W = 2 * self.Jo * self.NP, self._last - self._m0 + 1
        R1 = self.R + 1
        nk = self._nk[:R1].contiguous()
        nkb = self._nkb[:R1].contiguous()
        _lib.call("b3d_moments_flush", self.L, p(self._stage.m), p(self._stage.e), self._stage.m.stride(0),
                  p(self._row_shift), self._m0, W, rows, self.N, R1, p(nk), p(nkb), self.plan.order + 1, self._KW,
                  int(self._flushes > 0), self.Ld, p(self.mom.m), p(self.mom.e), self.mom.m.stride(0),
                  torch.cuda.current_stream(self.device).cuda_stream)
        self._flushes += 1
        self._last = None
        self._stage.e.fill_(mpf.EZ)                      # entries a level does not write read as zero

    # ------------------------------------------------------------ final GEMMs
    def finish(self, h_inf, chunk=None):
        """h_inf: MPF (2, order + 1, Jh, Smax^2, B).  Returns numerators MPF (Jo, Dout, R + 1, 2, Smax^2, B):
        [spin, x^k coefficient, log r derivative e, parity, structure a * Smax + b, rhs]"""
        return mpf.cat([num for _, num in self.finish_iter(h_inf, chunk)], 0)

    def finish_iter(self, h_inf, chunk=None):
        """as finish, by chunks of output spins: yields (first spin index, numerators)"""
        self.flush()
        R, Jo, NP, order, L, dev = self.R, self.Jo, self.NP, self.plan.order, self.Ld, self.device
        h_inf = resize(h_inf, L)
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
