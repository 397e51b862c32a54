// Index plan of the batched radial recursion (host C++): what the recursion kernels index with, built once per
// operator.  Replaces the reference's vectorised numpy builder recursion_gpu.Plan (recursion_gpu.py:136-365);
// the tensors it produces are the reference's (slot numbering, first-appearance key order, LIFO slot recycling),
// so that golden plans pin them, but the construction here is a single pass over the tasks of each level with
// hash maps for the first-appearance numberings and an explicit free-slot stack.
//
// blocks_3d's recursion (fill_residues.cxx) computes per level m one residue block per (parity p, spin tj, pole P):
//   H(src, m, tj', D') = h_inf[src][m][tj'] + sum_i 2 / (D' - D_i) res[src][m - shift_i][tj'][i]
//   res[p][m][tj][P]   = Q(P, tj) sign L_P H(src, m, tj', D'_P) R_P^T
// with tj' = child spin of P, D' = twice_position(P, tj) + 2 shift(P), src = (p + [P of type IV]) % 2.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "b3dgpu.h"

namespace b3d {
int fail(int code, const std::string& what);
}

namespace {

using i64 = int64_t;

i64 floordiv(i64 a, i64 b) { return a / b - ((a % b != 0) && ((a < 0) != (b < 0))); }
i64 posmod(i64 a, i64 b) { return ((a % b) + b) % b; }

// pole kinds 0..3 = blocks_3d's types I..IV (Pole_Types.cxx)
struct Kinds {
    i64 n[4];
    i64 total() const { return n[0] + n[1] + n[2] + n[3]; }
};

struct Spins {
    i64 tj12, tj43, tjmax;

    Kinds counts(i64 tj, i64 order) const {
        const i64 half = tj / 2, narrow = std::min(half, std::min(tj12 / 2, tj43 / 2));
        const bool boson = tj % 2 == 0;
        Kinds c{{order, std::min(half, order),
                 boson ? floordiv(order, 2) : std::min(narrow, floordiv(order, 2)),
                 boson ? std::min(narrow, floordiv(order + 1, 2)) : floordiv(order + 1, 2)}};
        for (i64& x : c.n) x = std::max<i64>(x, 0);
        return c;
    }
    // the idx-th pole of a block truncated at `order` (kind-major, k = 1, 2, ...)
    void pole_at(i64 tj, i64 order, i64 idx, i64& kind, i64& k) const {
        Kinds c = counts(tj, order);
        kind = 0;
        while (kind < 3 && idx >= c.n[kind]) idx -= c.n[kind++];
        k = idx + 1;
    }
    i64 index_of(i64 tj, i64 order, i64 kind, i64 k) const {
        Kinds c = counts(tj, order);
        i64 at = 0;
        for (i64 u = 0; u < kind; ++u) at += c.n[u];
        return at + k - 1;
    }
    i64 excess(i64 tj) const { return tj > tjmax ? (tj - tjmax) / 2 : 0; }
    static i64 shift(i64 kind, i64 k) { return kind < 2 ? k : (kind == 2 ? 2 * k : 2 * k - 1); }
    static i64 child(i64 kind, i64 k, i64 tj) { return kind == 0 ? tj + 2 * k : (kind == 1 ? tj - 2 * k : tj); }
    static i64 twice_pos(i64 kind, i64 k, i64 tj) {
        switch (kind) {
            case 0: return 2 - tj - 2 * k;
            case 1: return 4 + tj - 2 * k;
            case 2: return 3 - 2 * k;
            default: return 4 - 2 * k;
        }
    }
    // number of SO(3) structures of spins tj1 x tj2 with pseudo-parity pp (so3_tensor_parity.cxx)
    static i64 so3(i64 pp, i64 tj1, i64 tj2) {
        i64 n = 0;
        for (i64 c = std::abs(tj1 - tj2); c <= tj1 + tj2; c += 2) n += posmod(tj1 + tj2 - c - 2 * pp, 4) == 0;
        return n;
    }
};

// ids numbered in order of first appearance
struct Numbering {
    std::unordered_map<i64, i64> id;
    std::vector<i64> codes;
    i64 operator()(i64 code) {
        auto it = id.find(code);
        if (it != id.end()) return it->second;
        id.emplace(code, (i64)codes.size());
        codes.push_back(code);
        return (i64)codes.size() - 1;
    }
};

struct Level {
    i64 m = 0, nb = 0, Mr = 0, Kc = 0;
    std::vector<i64> gsrc, gj, col, rowd, nrow, cold, ncol;
    std::vector<i64> t_slot, t_hrow, t_L, t_R, t_q, t_qL, t_p, t_tj, t_kind, t_k;
};

}  // namespace

struct b3d_plan {
    Spins sp{};
    i64 order = 0, pp[2][2] = {{0, 0}, {0, 0}}, base = 0;
    i64 nspin = 0, Smax = 0, Jh = 0, nslots = 0, nphys = 0, zero_slot = 0, dmax = 1;
    std::vector<i64> nl[2], nr[2];           // structure counts per parity and spin index
    std::vector<i64> start, first;           // first logical slot of (m, spin index) = first[start[m] + ji]
    std::vector<i64> npol_flat;              // poles of (m, spin index), same indexing
    std::vector<Level> levels;               // nb == 0: no task at that level
    std::vector<i64> mkeys, qkeys, lqpairs;  // (kind, k, side, ppq, tj) / (kind, k, tj, sign) / (L id, Q id)
    std::vector<i64> phys;                   // logical -> physical slot, -1 where never written

    i64 ji(i64 tj) const { return (tj - base) / 2; }
    i64 nspins_at(i64 m) const {
        const i64 hi = sp.tjmax + 2 * (order - m - 1);
        return hi < base ? 0 : (hi - base) / 2 + 1;
    }

    void layout() {
        nspin = (sp.tjmax + 2 * order + 2 - base) / 2 + 1;
        for (int p = 0; p < 2; ++p) {
            nl[p].resize(nspin);
            nr[p].resize(nspin);
            for (i64 j = 0; j < nspin; ++j) {
                nl[p][j] = Spins::so3(pp[p][0], sp.tj12, base + 2 * j);
                nr[p][j] = Spins::so3(pp[p][1], sp.tj43, base + 2 * j);
            }
        }
        const i64 top = (sp.tjmax + 2 * order - base) / 2 + 1;
        for (int p = 0; p < 2; ++p)
            for (i64 j = 0; j < std::min(top, nspin); ++j) Smax = std::max({Smax, nl[p][j], nr[p][j]});
        Jh = top;
        i64 total = 0;
        for (i64 m = 0; m < order; ++m) {
            start.push_back((i64)first.size());
            for (i64 j = 0; j < nspins_at(m); ++j) {
                const i64 tj = base + 2 * j;
                const i64 n = sp.counts(tj, order - m - sp.excess(tj)).total();
                first.push_back(total);
                npol_flat.push_back(n);
                total += n;
            }
        }
        nslots = total;
        zero_slot = 2 * total;
    }

    // the tasks of level m and its Cauchy groups; keys are numbered afterwards over all levels
    void build_level(i64 m, Level& lv) {
        lv.m = m;
        Numbering groups;
        std::vector<std::vector<i64>> rows;                 // per group: its D' values in first-appearance order
        std::vector<std::unordered_map<i64, i64>> row_of;   // per group: D' -> row
        std::vector<i64> t_group, t_row;
        for (i64 j = 0; j < nspins_at(m); ++j) {
            const i64 tj = base + 2 * j, ord = order - m - sp.excess(tj), np = npol_flat[start[m] + j];
            for (i64 q = 0; q < np; ++q) {
                i64 kind, k;
                sp.pole_at(tj, ord, q, kind, k);
                const i64 tjc = Spins::child(kind, k, tj), jc = ji(tjc);
                const i64 dprime = Spins::twice_pos(kind, k, tj) + 2 * Spins::shift(kind, k);
                for (i64 p = 0; p < 2; ++p) {
                    const i64 src = (p + (kind == 3)) % 2;
                    if (!(nl[p][j] > 0 && nr[p][j] > 0 && nl[src][jc] > 0 && nr[src][jc] > 0)) continue;
                    const i64 g = groups(src * (i64(1) << 32) + tjc);
                    if (g == (i64)rows.size()) {
                        rows.emplace_back();
                        row_of.emplace_back();
                    }
                    auto it = row_of[g].find(dprime);
                    i64 r;
                    if (it == row_of[g].end()) {
                        r = (i64)rows[g].size();
                        row_of[g].emplace(dprime, r);
                        rows[g].push_back(dprime);
                    } else {
                        r = it->second;
                    }
                    lv.t_slot.push_back(p * nslots + first[start[m] + j] + q);
                    lv.t_p.push_back(p);
                    lv.t_tj.push_back(tj);
                    lv.t_kind.push_back(kind);
                    lv.t_k.push_back(k);
                    t_group.push_back(g);
                    t_row.push_back(r);
                }
            }
        }
        lv.nb = (i64)groups.codes.size();
        if (lv.nb == 0) return;
        for (auto& r : rows) lv.Mr = std::max(lv.Mr, (i64)r.size());
        lv.gsrc.resize(lv.nb);
        lv.gj.resize(lv.nb);
        lv.nrow.resize(lv.nb);
        lv.ncol.resize(lv.nb);
        lv.rowd.assign(lv.nb * lv.Mr, 0);
        for (i64 g = 0; g < lv.nb; ++g) {
            lv.gsrc[g] = groups.codes[g] >> 32;
            const i64 tjc = groups.codes[g] & 0xFFFFFFFF;
            lv.gj[g] = tjc / 2;
            lv.nrow[g] = (i64)rows[g].size();
            std::copy(rows[g].begin(), rows[g].end(), lv.rowd.begin() + g * lv.Mr);
            lv.ncol[g] = sp.counts(tjc, m).total();
            lv.Kc = std::max(lv.Kc, lv.ncol[g]);
        }
        lv.Kc = std::max<i64>(lv.Kc, 1);
        lv.col.assign(lv.nb * lv.Kc, zero_slot);
        lv.cold.assign(lv.nb * lv.Kc, 0);
        for (i64 g = 0; g < lv.nb; ++g) {
            const i64 tjc = groups.codes[g] & 0xFFFFFFFF;
            if (lv.ncol[g] == 0) continue;
            i64 cmin = INT64_MAX, cmax = INT64_MIN;
            for (i64 c = 0; c < lv.ncol[g]; ++c) {
                // column c: the c-th pole of tj' at order m, whose residue was made at level m - shift
                i64 kind, k;
                sp.pole_at(tjc, m, c, kind, k);
                const i64 sh = Spins::shift(kind, k), born = m - sh;
                const i64 pos = sp.index_of(tjc, order - born - sp.excess(tjc), kind, k);
                lv.col[g * lv.Kc + c] = lv.gsrc[g] * nslots + first[start[born] + ji(tjc)] + pos;
                const i64 d = Spins::twice_pos(kind, k, tjc);
                lv.cold[g * lv.Kc + c] = d;
                cmin = std::min(cmin, d);
                cmax = std::max(cmax, d);
            }
            const i64 rmin = *std::min_element(rows[g].begin(), rows[g].end());
            const i64 rmax = *std::max_element(rows[g].begin(), rows[g].end());
            dmax = std::max({dmax, std::abs(rmax - cmin), std::abs(rmin - cmax)});
        }
        lv.t_hrow.resize(t_group.size());
        for (size_t t = 0; t < t_group.size(); ++t) lv.t_hrow[t] = t_group[t] * lv.Mr + t_row[t];
    }

    // M matrix keys (L before R per task), Q keys and (L, Q) pairs, each numbered by first appearance
    void number_keys() {
        const i64 KM = order + 2, TJM = sp.tjmax + 2 * order + 4;
        const i64 PPM = std::max({pp[0][0], pp[0][1], pp[1][0], pp[1][1]}) + 1;
        Numbering mk, qk, lq;
        auto mcode = [&](i64 kind, i64 k, i64 side, i64 ppq, i64 tj) {
            return (((kind * KM + k) * 2 + side) * PPM + ppq) * TJM + tj;
        };
        for (Level& lv : levels) {
            const size_t T = lv.t_slot.size();
            lv.t_L.resize(T);
            lv.t_R.resize(T);
            lv.t_q.resize(T);
            for (size_t t = 0; t < T; ++t) {
                const i64 kind = lv.t_kind[t], k = lv.t_k[t], tj = lv.t_tj[t];
                const i64 src = (lv.t_p[t] + (kind == 3)) % 2;
                lv.t_L[t] = mk(mcode(kind, k, 0, pp[src][0], tj));
                lv.t_R[t] = mk(mcode(kind, k, 1, pp[src][1], tj));
                const i64 tjc = Spins::child(kind, k, tj);
                const bool positive = posmod(tjc - tj, 4) == 0;
                lv.t_q[t] = qk(((kind * KM + k) * TJM + tj) * 2 + positive);
            }
        }
        for (i64 c : mk.codes) {
            const i64 tj = c % TJM, ppq = (c / TJM) % PPM, side = (c / TJM / PPM) % 2, r = c / TJM / PPM / 2;
            mkeys.insert(mkeys.end(), {r / KM, r % KM, side, ppq, tj});
        }
        for (i64 c : qk.codes) {
            const i64 positive = c % 2, tj = (c / 2) % TJM, r = c / 2 / TJM;
            qkeys.insert(qkeys.end(), {r / KM, r % KM, tj, positive ? 1 : -1});
        }
        const i64 nq = (i64)qk.codes.size();
        for (Level& lv : levels) {
            lv.t_qL.resize(lv.t_slot.size());
            for (size_t t = 0; t < lv.t_slot.size(); ++t) lv.t_qL[t] = lq(lv.t_L[t] * nq + lv.t_q[t]);
        }
        for (i64 c : lq.codes) lqpairs.insert(lqpairs.end(), {c / nq, c % nq});
    }

    // Physical slots.  Without reuse, every written logical slot is its own physical slot.  With reuse, a slot
    // is released after the last level that reads it as a Cauchy column (a level gathers its columns before its
    // pole step writes, so that level's own outputs may take it), or after its own level if no level reads it.
    // Released slots go on a stack and are handed out from its top; at each level, the release batches that
    // have come due are pushed in the order their release levels were first scheduled, each batch in slot
    // order.  This is the allocation order of the reference builder, which the golden plans pin.
    void recycle(bool reuse) {
        const i64 nlog = 2 * nslots;
        std::vector<i64> born(nlog, -1), last(nlog, -1);
        for (const Level& lv : levels) {
            for (i64 s : lv.t_slot) born[s] = lv.m;
            for (i64 c : lv.col)
                if (c != zero_slot) last[c] = std::max(last[c], lv.m);
        }
        phys.assign(nlog, -1);
        if (!reuse) {
            for (i64 s = 0; s < nlog; ++s)
                if (born[s] >= 0) phys[s] = s;
            nphys = nlog;
        } else {
            std::vector<std::vector<i64>> by_level(order);
            for (i64 s = 0; s < nlog; ++s)
                if (born[s] >= 0) by_level[born[s]].push_back(s);
            std::vector<i64> stack;
            std::vector<i64> sched;                                  // release levels, in first-scheduled order
            std::unordered_map<i64, std::vector<i64>> batches;       // release level -> slots, pushed in order
            i64 used = 0;
            for (i64 m = 0; m < order; ++m) {
                const std::vector<i64>& seg = by_level[m];
                if (seg.empty()) continue;
                std::vector<i64> keep;
                for (i64 lvl : sched) {
                    if (lvl <= m) {
                        auto& b = batches[lvl];
                        stack.insert(stack.end(), b.begin(), b.end());
                        batches.erase(lvl);
                    } else {
                        keep.push_back(lvl);
                    }
                }
                sched.swap(keep);
                for (i64 s : seg) {
                    i64 ph;
                    if (!stack.empty()) {
                        ph = stack.back();
                        stack.pop_back();
                    } else {
                        ph = used++;
                    }
                    phys[s] = ph;
                    const i64 rel = last[s] > m ? last[s] : m + 1;
                    auto it = batches.find(rel);
                    if (it == batches.end()) {
                        sched.push_back(rel);
                        batches.emplace(rel, std::vector<i64>{ph});
                    } else {
                        it->second.push_back(ph);
                    }
                }
            }
            nphys = used;
        }
        zero_slot = nphys;
        const i64 old_zero = 2 * nslots;
        for (Level& lv : levels) {
            for (i64& s : lv.t_slot) s = phys[s];
            for (i64& c : lv.col) c = (c == old_zero || phys[c] < 0) ? nphys : phys[c];
        }
    }
};

namespace {
template <class V>
void put(const V& v, int64_t* dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int64_t));
}
}  // namespace

extern "C" {

int b3d_plan_build(int64_t two_j12, int64_t two_j43, int64_t two_j_max, int64_t order, const int64_t* pseudo_parities,
                   int reuse, b3d_plan** out) {
    if (!out || !pseudo_parities || two_j12 < 0 || two_j43 < 0 || two_j_max < 0 || order < 1)
        return b3d::fail(B3D_E_ARG, "b3d_plan_build: invalid arguments");
    if (two_j_max % 2 != two_j12 % 2 || two_j12 % 2 != two_j43 % 2)
        return b3d::fail(B3D_E_ARG, "b3d_plan_build: two_j_max, two_j12 and two_j43 must have one parity");
    for (int i = 0; i < 4; ++i)
        if (pseudo_parities[i] < 0 || pseudo_parities[i] > 1)
            return b3d::fail(B3D_E_ARG, "b3d_plan_build: pseudo-parities are 0 or 1");
    b3d_plan* pl = new (std::nothrow) b3d_plan;
    if (!pl) return b3d::fail(B3D_E_ARG, "b3d_plan_build: out of host memory");
    try {
        pl->sp = Spins{two_j12, two_j43, two_j_max};
        pl->order = order;
        pl->base = two_j12 % 2;
        for (int i = 0; i < 4; ++i) pl->pp[i / 2][i % 2] = pseudo_parities[i];
        pl->layout();
        pl->levels.resize(order);
        for (int64_t m = 0; m < order; ++m) pl->build_level(m, pl->levels[m]);
        pl->number_keys();
        pl->recycle(reuse != 0);
    } catch (const std::exception& e) {
        delete pl;
        return b3d::fail(B3D_E_ARG, std::string("b3d_plan_build: ") + e.what());
    }
    *out = pl;
    return 0;
}

void b3d_plan_destroy(b3d_plan* plan) { delete plan; }

int b3d_plan_scalars(const b3d_plan* pl, int64_t* s) {
    if (!pl || !s) return b3d::fail(B3D_E_ARG, "b3d_plan_scalars: null argument");
    const int64_t v[B3D_PLAN_NSCALARS] = {pl->Smax, pl->Jh, pl->nslots, pl->nphys, pl->zero_slot, pl->dmax,
                                          pl->order, (int64_t)pl->mkeys.size() / 5, (int64_t)pl->qkeys.size() / 4,
                                          (int64_t)pl->lqpairs.size() / 2, (int64_t)pl->first.size()};
    std::memcpy(s, v, sizeof v);
    return 0;
}

int b3d_plan_keys(const b3d_plan* pl, int64_t* mkeys, int64_t* qkeys, int64_t* lqpairs) {
    if (!pl) return b3d::fail(B3D_E_ARG, "b3d_plan_keys: null plan");
    put(pl->mkeys, mkeys);
    put(pl->qkeys, qkeys);
    put(pl->lqpairs, lqpairs);
    return 0;
}

int b3d_plan_layout(const b3d_plan* pl, int64_t* start, int64_t* first, int64_t* phys) {
    if (!pl) return b3d::fail(B3D_E_ARG, "b3d_plan_layout: null plan");
    put(pl->start, start);
    put(pl->first, first);
    put(pl->phys, phys);
    return 0;
}

int b3d_plan_level_dims(const b3d_plan* pl, int64_t m, int64_t* dims) {
    if (!pl || !dims || m < 0 || m >= pl->order) return b3d::fail(B3D_E_ARG, "b3d_plan_level_dims: bad level");
    const Level& lv = pl->levels[m];
    dims[0] = lv.nb;
    dims[1] = lv.Mr;
    dims[2] = lv.Kc;
    dims[3] = (int64_t)lv.t_slot.size();
    return 0;
}

int b3d_plan_level(const b3d_plan* pl, int64_t m, const b3d_plan_level_arrays* a) {
    if (!pl || !a || m < 0 || m >= pl->order) return b3d::fail(B3D_E_ARG, "b3d_plan_level: bad level");
    const Level& lv = pl->levels[m];
    put(lv.gsrc, a->gsrc);
    put(lv.gj, a->gj);
    put(lv.col, a->col);
    put(lv.rowd, a->rowd);
    put(lv.nrow, a->nrow);
    put(lv.cold, a->cold);
    put(lv.ncol, a->ncol);
    put(lv.t_slot, a->t_slot);
    put(lv.t_hrow, a->t_hrow);
    put(lv.t_L, a->t_L);
    put(lv.t_R, a->t_R);
    put(lv.t_q, a->t_q);
    put(lv.t_qL, a->t_qL);
    put(lv.t_p, a->t_p);
    put(lv.t_tj, a->t_tj);
    put(lv.t_kind, a->t_kind);
    put(lv.t_k, a->t_k);
    return 0;
}

}  // extern "C"
