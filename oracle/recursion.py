"""Oracle radial recursion: blocks_3d's fill_residues / set_residue, level by level, one (spin, pole,
parity) at a time, in mpmath.  Restates the reference's exact CPU port recursion_ref.py:11-44.
Test infrastructure only.

Inputs: h_inf[(src, m, jh, a, b)] and M[(pole, side, tjNN, ppq, tj)] -> matrix (list of rows) of mpmath
numbers; missing entries are zero.  Output: res[(p, m, jidx, pole index, a, b)].
"""
import mpmath as mp

from . import blocks as B


def fill_level(h_inf, M, res, m, tj12, tj43, tj_max, order, pseudo_parities, jsel=None, t_end=None):
    """the residues of level m (every spin index, or those in jsel), read from the residues of the levels
    below in res; returns (new residues, MACs done, completed before t_end)"""
    import time
    zero = mp.mpf(0)
    out, macs = {}, 0
    for jidx, tj in enumerate(B.spins(m, order, tj12, tj_max)):
        if jsel is not None and jidx not in jsel:
            continue
        for pidx, P in enumerate(B.pole_list(tj, tj12, tj43, order - m - B.excess(tj, tj_max))):
            tjc = B.child(P, tj)
            d_row = B.twice_pos(P, tj) + 2 * B.shift(P)
            exc = B.excess(tjc, tj_max)
            terms = []
            for i in B.pole_list(tjc, tj12, tj43, m):
                diff = d_row - B.twice_pos(i, tjc)
                coef = mp.mpf(2) / diff if diff else zero
                pos = B.pole_list(tjc, tj12, tj43, order - m + B.shift(i) - exc).index(i)
                terms.append((m - B.shift(i), pos, coef))
            q = B.q_value(P, tj)
            qv = mp.mpf(q.numerator) / q.denominator
            if (tjc - tj) % 4:
                qv = -qv
            for p in range(2):
                src = (p + (1 if P[0] == 3 else 0)) % 2
                left = M.get((P, 0, tj12, pseudo_parities[src][0], tj))
                right = M.get((P, 1, tj43, pseudo_parities[src][1], tj))
                if not left or not left[0] or not right or not right[0]:
                    continue
                nl, nr = len(left[0]), len(right[0])
                jc = tjc // 2
                h = [[h_inf.get((src, m, jc, a, b), zero)
                      + mp.fsum(res.get((src, mm, jc, pos, a, b), zero) * c for mm, pos, c in terms)
                      for b in range(nr)] for a in range(nl)]
                for a0 in range(len(left)):
                    for b0 in range(len(right)):
                        out[(p, m, jidx, pidx, a0, b0)] = qv * mp.fsum(
                            left[a0][a] * h[a][b] * right[b0][b] for a in range(nl) for b in range(nr))
                macs += len(terms) * nl * nr + 2 * len(left) * len(right) * nl * nr
            if t_end is not None and time.perf_counter() > t_end:
                return out, macs, False
    return out, macs, True


def fill_residues(h_inf, M, tj12, tj43, tj_max, order, pseudo_parities, budget=None, stats=None):
    """budget: stop after this many seconds (a bounded sample for CPU timing); stats: dict receiving the
    multiprecision MACs done ("macs") and whether the run completed ("complete")"""
    import time
    t_end = None if budget is None else time.perf_counter() + budget
    macs, done = 0, True
    res = {}
    for m in range(order):
        new, n, done = fill_level(h_inf, M, res, m, tj12, tj43, tj_max, order, pseudo_parities, t_end=t_end)
        res.update(new)
        macs += n
        if not done:
            break
    if stats is not None:
        stats.update(macs=macs, complete=done)
    return res


def count_macs(tj12, tj43, tj_max, order, pseudo_parities, M_shapes):
    """multiprecision MACs fill_residues does for one right-hand side (the count of its loops, no arithmetic);
    M_shapes[key] = (rows, cols) of the matrices present"""
    macs = 0
    for m in range(order):
        for jidx, tj in enumerate(B.spins(m, order, tj12, tj_max)):
            for P in B.pole_list(tj, tj12, tj43, order - m - B.excess(tj, tj_max)):
                nterms = len(B.pole_list(B.child(P, tj), tj12, tj43, m))
                for p in range(2):
                    src = (p + (1 if P[0] == 3 else 0)) % 2
                    ls = M_shapes.get((P, 0, tj12, pseudo_parities[src][0], tj))
                    rs = M_shapes.get((P, 1, tj43, pseudo_parities[src][1], tj))
                    if not ls or not rs or not ls[1] or not rs[1]:
                        continue
                    nl, nr = ls[1], rs[1]
                    macs += nterms * nl * nr + 2 * ls[0] * rs[0] * nl * nr
    return macs
