"""Batched radial recursion of blocks_3d on one B200: the host half of the reference's
``recursion_gpu.Recursion`` (``blocksvibe/recursion_gpu.py:379-514``), same constructor and ``run``
contract.

Per level m (a ``Plan`` level): one kernel for the Cauchy step fused with the h_inf term
(``b3d_cauchy_level``), one pair of kernels for the pole step writing straight into the slot buffer
(``b3d_pole_level_mma``: the exact sums as INT8 tensor-core GEMMs of base-256 digits; ``b3d_pole_level``: the
same bits on the CUDA cores), then the caller's hook (the derivative moments).  Constants are built once per
operator: the M-matrix table, the exact Q values with their sign, q L for every (L, Q) pair of the plan,
and the R and q L tables aligned per row for the pole step.
"""
from fractions import Fraction

import numpy as np
import torch

from . import _lib, mpf, structure as S
from .mpf import MPF


# default Cauchy kernel and pole-step kernel (see Recursion)
CAUCHY = "cuda4"
POLE = "auto"
# Which pole-step form is faster.  The tensor-core form takes a task's S B columns in chunks of 32 at a cost per
# chunk that hardly depends on how many columns are in use; the CUDA-core form costs in proportion to the
# columns.  Measured on a B200 (both forms, both stages, 3000 synthetic tasks per shape, L in {26, 30, 34, 42},
# S in {2 .. 5}, S B from 5 to 130): the time ratio CUDA cores / tensor cores of a full chunk, by (L, S); for other
# column counts the ratio scales with the chunks' fill (S B / (32 chunks)) to within a few percent.
POLE_FULL_CHUNK_RATIO = {26: (0.71, 0.91, 1.09, 1.23), 30: (0.64, 0.85, 1.02, 1.14), 34: (0.73, 0.93, 1.09, 1.24),
                         42: (0.90, 1.15, 1.32, 1.51)}            # S = 2, 3, 4, 5
POLE_MIN_GAIN = 1.05


def pole_mma_gain(L, S, B):
    """predicted time ratio CUDA-core / tensor-core pole step (above 1: the tensor cores are faster)"""
    if S < 2:
        return 0.0
    Lk = max((k for k in POLE_FULL_CHUNK_RATIO if k <= L), default=26)
    r = POLE_FULL_CHUNK_RATIO[Lk][min(S, 5) - 2]
    cols = S * B
    return r * cols / (32 * -(-cols // 32))


def _dev(a, device):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int64).to(device)


class Recursion:
    """Numbers of one Plan on the GPU.  M: dict key -> matrix of decimal strings (keys as plan.Mkeys),
    an MPF table (nM, Smax, Smax) in plan.Mkeys order, or None for random O(1) matrices (timing runs)."""

    def __init__(self, plan, M, L, device="cuda", generator=None, cauchy=None, rns_min_k=32, pole=None):
        """cauchy: "cuda" (one-limb divisions on the CUDA cores, b3d_cauchy_level), "cuda2" (the same quotients from
        pre-aligned columns, two per thread, b3d_cauchy_align + b3d_cauchy_level2: bit-identical to "cuda"), "cuda3"
        (cuda2 with 24- or 22-bit quotient digits when the plan's divisors allow, b3d_cauchy_level3: bit-identical), "cuda4"
        (cuda3 on sign-magnitude columns read limb by limb, b3d_cauchy_align_sm + b3d_cauchy_level4: bit-identical), "rns"
        (the level's Cauchy GEMM on the tensor cores, residues + CRT), or "auto" (rns for levels with at least
        rns_min_k columns, cuda2 below).  pole: "mma" (the pole step's exact sums on the INT8 tensor cores,
        b3d_pole_level_mma; plans with Smax <= 8), "cuda" (b3d_pole_level) or "auto" (mma where the measured
        crossover, pole_mma_gain, predicts it faster, cuda elsewhere): bit-identical"""
        self.cauchy, self.rns_min_k = cauchy or CAUCHY, rns_min_k
        self.pole = pole or POLE
        if self.pole not in ("mma", "cuda", "auto"):
            raise ValueError(f"pole must be 'mma', 'cuda' or 'auto', not {self.pole!r}")
        if self.pole != "cuda" and plan.Smax > 8:
            self.pole = "cuda"
        self._side = {}                                  # calling stream -> stream of the per-level hook
        self.overlap_hook = True
        if not _lib.lib().b3d_supported_limbs(L):
            raise _lib.B3DError(f"no kernels compiled for L = {L}")
        if plan.dmax >= 1 << 16:
            raise _lib.B3DError(f"Cauchy differences up to {plan.dmax} exceed the one-limb kernel (< 65536)")
        self.plan, self.L, self.device = plan, L, torch.device(device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)   # bounded-wait expiries of the kernels
        Sm, nM = plan.Smax, len(plan.Mkeys)
        if M is None:
            self.Mtab = mpf.random_mpf((nM, Sm, Sm), L, spread=1, device=self.device, generator=generator)
        elif isinstance(M, MPF):
            self.Mtab = M.to(self.device)
        else:
            strs = ["0"] * (nM * Sm * Sm)
            for key, i in plan.Mkeys.items():
                for a, row in enumerate(M.get(key) or []):
                    for b, x in enumerate(row):
                        strs[(i * Sm + a) * Sm + b] = x
            self.Mtab = mpf.from_strings(strs, L, (nM, Sm, Sm), self.device)
        self._constants()

    def _constants(self):
        plan, L, dev, Sm = self.plan, self.L, self.device, self.plan.Smax
        qv = [Fraction(0)] * len(plan.Qkeys)
        for (P, tj, sign), i in plan.Qkeys.items():
            qv[i] = S.residue_prefactor(P, tj) * sign
        self.Qtab = mpf.from_fractions(qv, L, (len(qv),), dev)
        nlq = len(plan.LQpairs)
        pairs = torch.as_tensor(plan.LQpairs, dtype=torch.int64, device=dev).reshape(nlq, 2)
        s2 = torch.arange(Sm * Sm, device=dev)
        aidx = (pairs[:, 0:1] * Sm * Sm + s2).reshape(-1)
        bidx = pairs[:, 1:2].expand(nlq, Sm * Sm).reshape(-1)
        QL = mpf.mul(self.Mtab.reshape(-1), self.Qtab, aidx=aidx, bidx=bidx, shape=(nlq, Sm, Sm))
        self.Ralign = mpf.align_rows(self.Mtab)        # (L, nM, S, S), (nM, S)
        self.QLalign = mpf.align_rows(QL)
        self.levels = []
        for lev in plan.levels:
            if lev is None:
                self.levels.append(None)
                continue
            d = {k: _dev(lev[k], dev) for k in ("gsrc", "gj", "rowd", "nrow", "cold", "ncol", "col",
                                                   "t_slot", "t_hrow", "t_R", "t_qL")}
            d.update(m=lev["m"], nb=lev["nb"], Mr=lev["Mr"], Kc=lev["Kc"], T=len(lev["t_slot"]))
            self.levels.append(d)
        live = [d for d in self.levels if d]
        self.max_rows = max((d["nb"] * d["Mr"] for d in live), default=0)
        self.max_tasks = max((d["T"] for d in live), default=0)
        self._ctable = None

    def _cauchy_table(self):
        """residues of round(2^(NB-1) / d), |d| <= dmax, per prime: (2 dmax + 1, np) on the device"""
        if self._ctable is None:
            from . import rns
            tb = rns.tables(self.L, self.device)
            ps = [int(x) & 0xFFFFFFFF for x in tb.p.cpu().tolist()]
            NB, dm = mpf.nbits(self.L), self.plan.dmax
            rows = []
            for d in range(-dm, dm + 1):
                if d == 0:
                    rows.append([0] * len(ps))
                    continue
                a = abs(d)
                q = ((1 << (NB - 1)) + a // 2) // a          # round half up on the magnitude
                v = -q if d < 0 else q
                rows.append([v % p for p in ps])
            self._ctable = torch.tensor(np.array(rows, dtype=np.uint32).view(np.int32), device=self.device)
        return self._ctable

    def _use_rns(self, lev):
        if self.cauchy in ("cuda", "cuda2", "cuda3", "cuda4") or lev["m"] == 0 or lev["Kc"] > 256:
            return False
        return self.cauchy == "rns" or lev["Kc"] >= self.rns_min_k

    def _cauchy_rns(self, lev, tabs, res, h_inf, H, stream):
        """the level's Cauchy step as RNS GEMMs on the tensor cores, then + h_inf: H (nb Mr, N)"""
        import ctypes
        from . import rns
        L, dev = self.L, self.device
        nb, Mr, Kc, N = lev["nb"], lev["Mr"], lev["Kc"], tabs.N
        p = lambda t: t.data_ptr()
        tb = rns.tables(L, dev)
        Xm = torch.empty((L, nb * Kc * N), dtype=torch.int32, device=dev)
        Xe = torch.empty((nb, N), dtype=torch.int64, device=dev)
        _lib.call("b3d_cauchy_align", L, p(res.m), p(res.e), res.m.stride(0), _lib.ctypes_byref(tabs), p(Xm), p(Xe),
                  Xm.stride(0), stream)
        Kp = -(-Kc // 32) * 32
        table = self._cauchy_table()
        c_rows = Mr >= N                                           # C on the 128 TMEM lanes
        TN = min(256, -(-4 * (N if c_rows else Mr) // 16) * 16)
        TRc = 128 if c_rows else TN
        Rp_c = -(-Mr // (TRc // 4)) * (TRc // 4)
        c_mat = 4 * Rp_c * Kp
        C = torch.empty(tb.np * nb * c_mat, dtype=torch.uint8, device=dev)
        _lib.call("b3d_cauchy_digits", _lib.ctypes_byref(tabs), p(table), self.plan.dmax, tb.np, Rp_c, Kp, TRc, c_mat,
                  p(C), stream)
        X, x_mat, Rp_x = rns._split(tb, Xm, Xm.stride(0), nb, N, Kc, Kc * N, 1, N, Kp, TN if c_rows else 128, stream)
        if c_rows:
            A, a_mat, B8, b_mat, NI, NL, Rp_l, oi, ol = C, c_mat, X, x_mat, Mr, N, Rp_x, N, 1
        else:
            A, a_mat, B8, b_mat, NI, NL, Rp_l, oi, ol = X, x_mat, C, c_mat, N, Mr, Rp_c, 1, N
        n = nb * Mr * N
        # the CRT operand's padding columns meet zero rows of the constant matrix: no clearing needed
        yb = torch.empty((-(-n // 128) * 128) * tb.Kc, dtype=torch.uint8, device=dev)
        args = rns.RnsMmaArgs(p(A), p(B8), a_mat, b_mat, nb, NI, NL, Kp, TN, (4 * Rp_l) // TN, Mr * N, oi, ol,
                              None, p(tb.err), p(yb), tb.Kc)
        rns._check(rns._bind().b3d_rns_mma(ctypes.byref(args), ctypes.byref(tb.c), stream), "b3d_rns_mma")
        Hm = torch.empty((L, n), dtype=torch.int32, device=dev)
        He = torch.empty(n, dtype=torch.int64, device=dev)
        ea = torch.full((nb, Mr), 2 - mpf.nbits(L), dtype=torch.int64, device=dev)
        cargs = rns.RnsCrtArgs(p(yb), p(tb.T), tb.Kc, tb.NH, n, nb, Mr, N, p(ea), p(Xe), p(Hm), p(He), Hm.stride(0),
                               p(tb.err))
        rns._check(rns._bind().b3d_rns_crt_mma(L, ctypes.byref(cargs), ctypes.byref(tb.c), stream), "b3d_rns_crt_mma")
        _lib.call("b3d_cauchy_add_hinf", L, p(Hm), p(He), Hm.stride(0), p(h_inf.m), p(h_inf.e), h_inf.m.stride(0),
                  _lib.ctypes_byref(tabs), p(H.m), p(H.e), H.m.stride(0), stream)

    def footprint_bytes(self, B):
        """device bytes run() allocates for B right-hand sides (slots, Cauchy rows, pole scratch)"""
        per = (4 * self.L + 8) * self.plan.Smax ** 2 * B
        return per * (self.plan.nphys + 1 + self.max_rows + self.max_tasks)

    def run(self, h_inf, hook=None, overlap=None):
        """h_inf: MPF (2, >= order, Jh, Smax^2, B).  Returns the residue slots MPF (nphys + 1, Smax^2, B);
        hook(m, res) runs after each level (e.g. Derivs.accumulate).  overlap: the hook of level m runs on a
        second stream, concurrently with the Cauchy step of level m + 1 (which only reads the slots and writes
        H); the pole step of level m + 1, which writes slots, waits for it.  None: self.overlap_hook."""
        plan, L, Sm = self.plan, self.L, self.plan.Smax
        S2, B = Sm * Sm, h_inf.shape[-1]
        N = S2 * B
        hlevels = h_inf.shape[1]
        if h_inf.L != L or h_inf.shape[2] < plan.Jh or hlevels < plan.order or h_inf.shape[3] != S2:
            raise ValueError(f"h_inf shape {h_inf.shape} (L={h_inf.L}) does not match the plan")
        h_inf = h_inf.contiguous()
        Jh = h_inf.shape[2]
        dev = self.device
        res = mpf.zeros((plan.nphys + 1, S2, B), L, dev)
        H = mpf.zeros((max(1, self.max_rows), N), L, dev)
        Y = mpf.zeros((max(1, self.max_tasks), S2, B), L, dev)
        main = torch.cuda.current_stream(dev)
        stream = main.cuda_stream
        side = None
        if overlap is None:
            overlap = self.overlap_hook
        if hook is not None and overlap:
            side = self._side.get(stream)
            if side is None:
                side = self._side[stream] = torch.cuda.Stream(dev)
        pending = None                                   # the side stream's last hook, not yet joined
        use_mma = self.uses_mma(B)
        p = lambda t: t.data_ptr()
        for lev in self.levels:
            if lev is None:
                continue
            tabs = _lib.LevelTables(lev["m"], lev["nb"], lev["Mr"], lev["Kc"], N, hlevels, Jh,
                                    p(lev["gsrc"]), p(lev["gj"]), p(lev["rowd"]), p(lev["nrow"]),
                                    p(lev["cold"]), p(lev["ncol"]), p(lev["col"]))
            if self._use_rns(lev):
                self._cauchy_rns(lev, tabs, res, h_inf, H, stream)
            elif self.cauchy == "cuda4" and lev["m"] > 0:
                nb, Kc = lev["nb"], lev["Kc"]
                Xm = torch.empty((L, nb * Kc * N), dtype=torch.int32, device=dev)
                Xe = torch.empty((nb, N), dtype=torch.int64, device=dev)
                _lib.call("b3d_cauchy_align_sm", L, p(res.m), p(res.e), res.m.stride(0), _lib.ctypes_byref(tabs), p(Xm),
                          p(Xe), Xm.stride(0), stream)
                _lib.call("b3d_cauchy_level4", L, p(Xm), p(Xe), Xm.stride(0), p(h_inf.m), p(h_inf.e),
                          h_inf.m.stride(0), _lib.ctypes_byref(tabs), plan.dmax, p(H.m), p(H.e), H.m.stride(0), stream)
            elif self.cauchy in ("cuda2", "cuda3") and lev["m"] > 0:
                nb, Kc = lev["nb"], lev["Kc"]
                Xm = torch.empty((L, nb * Kc * N), dtype=torch.int32, device=dev)
                Xe = torch.empty((nb, N), dtype=torch.int64, device=dev)
                _lib.call("b3d_cauchy_align", L, p(res.m), p(res.e), res.m.stride(0), _lib.ctypes_byref(tabs), p(Xm),
                          p(Xe), Xm.stride(0), stream)
                if self.cauchy == "cuda3":
                    _lib.call("b3d_cauchy_level3", L, p(Xm), p(Xe), Xm.stride(0), p(h_inf.m), p(h_inf.e),
                              h_inf.m.stride(0), _lib.ctypes_byref(tabs), plan.dmax, p(H.m), p(H.e), H.m.stride(0), stream)
                else:
                    _lib.call("b3d_cauchy_level2", L, p(Xm), p(Xe), Xm.stride(0), p(h_inf.m), p(h_inf.e),
                              h_inf.m.stride(0), _lib.ctypes_byref(tabs), p(H.m), p(H.e), H.m.stride(0), stream)
            else:
                _lib.call("b3d_cauchy_level", L, p(res.m), p(res.e), res.m.stride(0), p(h_inf.m), p(h_inf.e),
                          h_inf.m.stride(0), _lib.ctypes_byref(tabs), p(H.m), p(H.e), H.m.stride(0), stream)
            if pending is not None:                      # slots written below may still be read by the hook
                main.wait_event(pending)
                pending = None
            pole_args = (L, p(H.m), p(H.e), H.m.stride(0),
                         p(self.Ralign[0]), p(self.Ralign[1]), self.Ralign[0].stride(0),
                         p(self.QLalign[0]), p(self.QLalign[1]), self.QLalign[0].stride(0),
                         p(lev["t_hrow"]), p(lev["t_R"]), p(lev["t_qL"]), p(lev["t_slot"]), lev["T"], B, Sm,
                         p(Y.m), p(Y.e), Y.m.stride(0), p(res.m), p(res.e), res.m.stride(0))
            if use_mma:
                _lib.call("b3d_pole_level_mma", *pole_args, p(self.err), stream)
            else:
                _lib.call("b3d_pole_level", *pole_args, stream)
            if hook is not None and side is not None:
                ready = torch.cuda.Event()
                ready.record(main)
                side.wait_event(ready)
                with torch.cuda.stream(side):
                    hook(lev["m"], res)
                pending = torch.cuda.Event()
                pending.record(side)
            elif hook is not None:
                hook(lev["m"], res)
        if pending is not None:
            main.wait_event(pending)
        return res

    def uses_mma(self, B):
        """whether run() with B right-hand sides takes the tensor-core pole step"""
        if self.pole != "auto":
            return self.pole == "mma"
        return pole_mma_gain(self.L, self.plan.Smax, B) >= POLE_MIN_GAIN

    def check_errors(self):
        """raise B3DError if a kernel of this recursion gave up a bounded wait (synchronises the device)"""
        code = int(self.err.item())
        if code:
            self.err.zero_()
            raise _lib.B3DError(f"pole step: a bounded wait of the tensor-core kernel expired (code {code})")

    def slot(self, p, m, jidx, pidx):
        """physical slot of residue (p, m, jidx, pidx) (meaningful after run() only without slot reuse)"""
        return self.plan.phys_slot(p * self.plan.nslots + self.plan.offset(m, jidx) + pidx)
