"""Index plan of the batched radial recursion for one operator (host side, numpy).

The recursion of blocks_3d (fill_residues.cxx) computes, level by level in m, one residue block per
(parity p, spin tj, pole P)::

    H(src, m, tj', D')   = h_inf[src][m][tj'] + sum_i 2 / (D' - D_i) res[src][m - shift_i][tj'][i]
    res[p][m][tj][P]     = Q(P, tj) sign L_P H(src, m, tj', D'_P) R_P^T

with tj' = child_spin(P, tj), D' = twice_position(P, tj) + 2 shift(P), src = (p + parity(P)) % 2.
The operator (pole positions, Cauchy coefficients, L/R matrices, Q) does not depend on the right-hand
side, so the whole index structure is built once here:

* a *logical slot* per residue block: ``p * nslots + first(m, jidx) + pole index``;
* per level, the Cauchy *groups* (src, tj') in order of first appearance, their *rows* (distinct D'),
  their *columns* (the prime poles i of tj' at order m and the slots holding their residues);
* per pole-step *task* its output slot, its H row, its L / R matrix keys, its Q key and its (L, Q)
  pair; keys are numbered in order of first appearance over all levels;
* optionally (``reuse=True``) a physical slot per logical one, recycled LIFO after the last level that
  reads it as a Cauchy column.

All tensors are identical to those of the reference builder ``recursion_gpu.Plan``
(``blocksvibe/recursion_gpu.py:136-365``), whose conventions the parity tests pin through golden
fixtures; the code is a separate implementation.
"""
import numpy as np

from . import structure as S


def first_appearance(codes):
    """(id of each code, distinct codes), ids numbered by first appearance"""
    codes = np.asarray(codes).reshape(-1)
    uniq, first, inverse = np.unique(codes, return_index=True, return_inverse=True)
    by_first = np.argsort(first, kind="stable")
    rank = np.empty(len(uniq), dtype=np.int64)
    rank[by_first] = np.arange(len(uniq))
    return rank[inverse.reshape(-1)], uniq[by_first]


class Plan:
    """Index plan for (tj12, tj43, tj_max, order, pseudo_parities); mirrors the reference ``Plan``
    (``recursion_gpu.py:136``): same constructor arguments and attribute names."""

    def __init__(self, two_j12, two_j43, two_j_max, order, pseudo_parities, reuse=False):
        self.tj12, self.tj43, self.tjmax, self.order = two_j12, two_j43, two_j_max, order
        self.pp = tuple(tuple(x) for x in pseudo_parities)
        self.base = two_j12 % 2
        nspin = (two_j_max + 2 * order + 2 - self.base) // 2 + 1       # every spin a task can touch
        spins = self.base + 2 * np.arange(nspin)
        self.nl = np.array([[len(S.so3_structures(self.pp[p][0], two_j12, int(t))) for t in spins] for p in (0, 1)])
        self.nr = np.array([[len(S.so3_structures(self.pp[p][1], two_j43, int(t))) for t in spins] for p in (0, 1)])
        top = (two_j_max + 2 * order - self.base) // 2 + 1
        self.Smax = int(max(self.nl[:, :top].max(), self.nr[:, :top].max()))
        self.Jh = len(S.level_spins(0, order + 1, two_j12, two_j_max))
        self._layout()
        self.dmax = 1
        raw = [self._level(m) for m in range(order)]
        self._number_keys(raw)
        self.levels = [None if r is None else r[0] for r in raw]
        self._assign_physical(reuse)

    def SL(self, p, tj):
        return int(self.nl[p, (tj - self.base) // 2])

    def SR(self, p, tj):
        return int(self.nr[p, (tj - self.base) // 2])

    # ------------------------------------------------------------ logical slot layout
    def _layout(self):
        self._tjs, self._ords, self._npol = [], [], []
        start, firsts, total, nent = [], [], 0, 0
        for m in range(self.order):
            tjs = np.arange(self.base, self.tjmax + 2 * (self.order - m - 1) + 1, 2, dtype=np.int64)
            ords = self.order - m - S.spin_excess_v(tjs, self.tjmax)
            npol = S.kind_counts_v(tjs, self.tj12, self.tj43, ords).sum(0)
            start.append(nent)
            nent += len(tjs)
            firsts.append(total + np.cumsum(npol) - npol)
            total += int(npol.sum())
            self._tjs.append(tjs)
            self._ords.append(ords)
            self._npol.append(npol)
        self._start = np.array(start, dtype=np.int64)
        self._flat = np.concatenate(firsts) if firsts else np.zeros(0, np.int64)
        self.nslots = total
        self.zero_slot = 2 * total

    def offset(self, m, jidx):
        """first logical slot of spin index jidx at level m (parity 0)"""
        return int(self._flat[self._start[m] + jidx])

    # ------------------------------------------------------------ one level
    def _level(self, m):
        tj12, tj43, ns = self.tj12, self.tj43, self.nslots
        tjs, ords, npol = self._tjs[m], self._ords[m], self._npol[m]
        ntot = int(npol.sum())
        if ntot == 0:
            return None
        jidx = np.repeat(np.arange(len(tjs)), npol)
        pidx = np.arange(ntot) - np.repeat(np.cumsum(npol) - npol, npol)
        tj = tjs[jidx]
        kind, k = S.pole_at_v(tj, tj12, tj43, ords[jidx], pidx)
        # both parities of each (spin, pole), parity innermost
        jidx, pidx, tj, kind, k = (np.repeat(a, 2) for a in (jidx, pidx, tj, kind, k))
        p = np.tile(np.array([0, 1], dtype=np.int64), ntot)
        tjp = S.child_spin_v(kind, k, tj)
        dprime = S.twice_position_v(kind, k, tj) + 2 * S.level_shift_v(kind, k)
        src = (p + (kind == S.KIND_IV)) % 2
        ji, jp = (tj - self.base) // 2, (tjp - self.base) // 2
        ok = (self.nl[p, ji] > 0) & (self.nr[p, ji] > 0) & (self.nl[src, jp] > 0) & (self.nr[src, jp] > 0)
        if not ok.any():
            return None
        jidx, pidx, tj, kind, k, p, tjp, dprime, src = (a[ok] for a in (jidx, pidx, tj, kind, k, p, tjp, dprime, src))
        slot = p * ns + self._flat[self._start[m] + jidx] + pidx

        # Cauchy groups (src, tj') and their rows D', numbered by first appearance
        gid, gcodes = first_appearance(src * (1 << 32) + tjp)
        nb = len(gcodes)
        gsrc, gtjp = gcodes >> 32, gcodes & 0xFFFFFFFF
        dlow = int(dprime.min())
        rid, rcodes = first_appearance(gid * (1 << 32) + (dprime - dlow))
        rgroup = rcodes >> 32
        by_group = np.argsort(rgroup, kind="stable")
        nrow = np.bincount(rgroup, minlength=nb)
        row_in_group = np.empty(len(rcodes), dtype=np.int64)
        row_in_group[by_group] = np.arange(len(rcodes)) - np.repeat(np.cumsum(nrow) - nrow, nrow)
        row = row_in_group[rid]
        Mr = int(nrow.max())
        rowd = np.zeros((nb, Mr), dtype=np.int64)
        rowd[rgroup, row_in_group] = (rcodes & 0xFFFFFFFF) + dlow

        # columns: the prime poles of tj' at order m, whose residues were produced at level m - shift
        ncol = S.kind_counts_v(gtjp, tj12, tj43, m).sum(0)
        Kc = max(1, int(ncol.max()))
        cg = np.repeat(np.arange(nb), ncol)
        cc = np.arange(int(ncol.sum())) - np.repeat(np.cumsum(ncol) - ncol, ncol)
        ctj = gtjp[cg]
        ckind, ck = S.pole_at_v(ctj, tj12, tj43, m, cc)
        csh = S.level_shift_v(ckind, ck)
        cslot = (gsrc[cg] * ns + self._flat[self._start[m - csh] + (ctj - self.base) // 2]
                 + S.pole_index_v(ctj, tj12, tj43, self.order - m + csh - S.spin_excess_v(ctj, self.tjmax), ckind, ck))
        col = np.full((nb, Kc), self.zero_slot, dtype=np.int64)
        col[cg, cc] = cslot
        cold = np.zeros((nb, Kc), dtype=np.int64)
        cold[cg, cc] = S.twice_position_v(ckind, ck, ctj)
        if len(cg):
            big = np.iinfo(np.int64).max
            cmin = np.full(nb, big); np.minimum.at(cmin, cg, cold[cg, cc])
            cmax = np.full(nb, -big); np.maximum.at(cmax, cg, cold[cg, cc])
            valid = np.arange(Mr)[None] < nrow[:, None]
            rmin = np.where(valid, rowd, big).min(1)
            rmax = np.where(valid, rowd, -big).max(1)
            has = ncol > 0
            if has.any():
                self.dmax = max(self.dmax, int(np.abs(rmax[has] - cmin[has]).max()),
                                int(np.abs(rmin[has] - cmax[has]).max()))
        sign = np.where((tjp - tj) % 4 != 0, -1, 1)
        ppa = np.array(self.pp, dtype=np.int64)
        lev = {"m": m, "nb": nb, "Mr": Mr, "Kc": Kc, "gsrc": gsrc, "gj": gtjp // 2, "col": col,
               "rowd": rowd, "nrow": nrow, "cold": cold, "ncol": ncol, "t_slot": slot, "t_hrow": gid * Mr + row}
        return lev, (kind, k, tj, ppa[src, 0], ppa[src, 1], sign)

    # ------------------------------------------------------------ M / Q / (L, Q) keys
    def _number_keys(self, raw):
        keyed = [r[1] for r in raw if r is not None]
        if not keyed:
            self.Mkeys, self.Qkeys, self.LQpairs = {}, {}, np.zeros((0, 2), np.int64)
            return
        kind, k, tj, ppl, ppr, sign = (np.concatenate([x[i] for x in keyed]) for i in range(6))
        KM, TJM = self.order + 2, self.tjmax + 2 * self.order + 4
        PPM = int(np.array(self.pp).max()) + 1

        def mcode(side, ppq):
            return (((kind * KM + k) * 2 + side) * PPM + ppq) * TJM + tj

        mid, mu = first_appearance(np.stack([mcode(0, ppl), mcode(1, ppr)], 1))
        tj_u, rest = mu % TJM, mu // TJM
        pq_u, rest = rest % PPM, rest // PPM
        side_u, rest = rest % 2, rest // 2
        k_u, kind_u = rest % KM, rest // KM
        self.Mkeys = {((int(a), int(b)), int(d), self.tj12 if d == 0 else self.tj43, int(c), int(t)): i
                      for i, (a, b, d, c, t) in enumerate(zip(kind_u, k_u, side_u, pq_u, tj_u))}
        qid, qu = first_appearance(((kind * KM + k) * TJM + tj) * 2 + (sign > 0))
        s_u, rest = qu % 2, qu // 2
        tjq_u, rest = rest % TJM, rest // TJM
        self.Qkeys = {((int(r // KM), int(r % KM)), int(t), 1 if s else -1): i
                      for i, (r, t, s) in enumerate(zip(rest, tjq_u, s_u))}
        nq = len(self.Qkeys)
        lqid, lqu = first_appearance(mid[0::2] * nq + qid)
        self.LQpairs = np.stack([lqu // nq, lqu % nq], 1)
        o = 0
        for r in raw:
            if r is None:
                continue
            lev, n = r[0], len(r[1][0])
            lev["t_L"] = mid[2 * o:2 * (o + n):2].copy()
            lev["t_R"] = mid[2 * o + 1:2 * (o + n):2].copy()
            lev["t_q"] = qid[o:o + n].copy()
            lev["t_qL"] = lqid[o:o + n].copy()
            o += n

    # ------------------------------------------------------------ physical slots
    def _assign_physical(self, reuse):
        """logical -> physical slot map (-1: never written, reads as the zero slot).  With reuse a slot is
        freed after the last level that reads it as a Cauchy column (the level's columns are gathered
        before its pole step writes), or after its own level if nothing reads it; freed slots are handed
        out last-in first-out, in the allocation order of the reference builder."""
        nlog, zero = 2 * self.nslots, self.zero_slot
        born = np.full(nlog, -1, dtype=np.int64)
        last = np.full(nlog, -1, dtype=np.int64)
        for lev in self.levels:
            if lev is None:
                continue
            born[lev["t_slot"]] = lev["m"]
            c = lev["col"].reshape(-1)
            np.maximum.at(last, c[c != zero], lev["m"])
        phys = np.full(nlog, -1, dtype=np.int64)
        if not reuse:
            live = born >= 0
            phys[live] = np.flatnonzero(live)
            self.nphys = nlog
        else:
            seq = np.argsort(born, kind="stable")
            seq = seq[born[seq] >= 0]
            cuts = np.flatnonzero(np.diff(born[seq])) + 1
            free = np.zeros(0, dtype=np.int64)
            pending = {}                       # release level -> list of slot arrays (insertion ordered)
            used = 0
            for seg in np.split(seq, cuts):
                if not len(seg):
                    continue
                m = int(born[seg[0]])
                due = [lvl for lvl in pending if lvl <= m]
                if due:
                    free = np.concatenate([free] + [a for lvl in due for a in pending.pop(lvl)])
                take = min(len(seg), len(free))
                got = np.empty(len(seg), dtype=np.int64)
                got[:take] = free[len(free) - take:][::-1]
                got[take:] = used + np.arange(len(seg) - take)
                used += len(seg) - take
                free = free[:len(free) - take]
                phys[seg] = got
                rel = np.where(last[seg] > m, last[seg], m + 1)
                _, first = np.unique(rel, return_index=True)
                for lvl in rel[np.sort(first)]:
                    pending.setdefault(int(lvl), []).append(got[rel == lvl])
            self.nphys = used
        self.phys = phys
        self.zero_slot = self.nphys
        for lev in self.levels:
            if lev is None:
                continue
            lev["t_slot"] = phys[lev["t_slot"]]
            c = lev["col"]
            mapped = np.full(c.shape, self.nphys, dtype=np.int64)
            real = c != zero
            mapped[real] = phys[c[real]]
            lev["col"] = np.where(mapped >= 0, mapped, self.nphys)

    def phys_slots(self, logical):
        """physical slots of logical ones (the zero slot where never written)"""
        logical = np.asarray(logical, dtype=np.int64)
        inside = logical < len(self.phys)
        p = self.phys[np.where(inside, logical, 0)]
        return np.where(inside & (p >= 0), p, self.zero_slot)

    def phys_slot(self, logical):
        return int(self.phys_slots(np.array([logical]))[0])

    def counts(self):
        """(Cauchy output entries, pole-step output entries) per right-hand side, rows padded per level
        and structures padded to Smax^2 (reference ``recursion_gpu.py:360``)"""
        s2 = self.Smax ** 2
        h = sum(lev["nb"] * lev["Mr"] for lev in self.levels if lev) * s2
        r = sum(len(lev["t_slot"]) for lev in self.levels if lev) * s2
        return h, r


def cauchy_tables(lev):
    """dense per-level Cauchy tables from row / column pole positions: cdiff = D' - D_i (0 for padding
    and coinciding positions) and cidx (0 -> zero, 2k - 1 -> +2/k, 2k -> -2/k)
    (reference ``recursion_gpu.py:368-376``)"""
    vr = np.arange(lev["Mr"])[None] < lev["nrow"][:, None]
    vc = np.arange(lev["Kc"])[None] < lev["ncol"][:, None]
    diff = np.where(vr[:, :, None] & vc[:, None, :], lev["rowd"][:, :, None] - lev["cold"][:, None, :], 0)
    cidx = np.where(diff == 0, 0, 2 * np.abs(diff) - (diff > 0))
    return diff.astype(np.int32), cidx.astype(np.int64)
