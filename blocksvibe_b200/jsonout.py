"""blocks_3d's per-spin JSON files, formatted on the GPU.  Replaces the reference's writer for the drop-in's
results (``cli._write`` / ``_write_one``, ``cli.py:453-490``, and ``b3djson.write_spin``, ``b3djson.py:97-198``):
the same bytes, with every number printed by the GPU instead of one MPFR conversion per number on the CPU.

    text = SpinWriter(opts, tjs, pp, outputs, Smax, nq, Dmax).render(device_outputs, q)   # {two_j: bytes}

``opts`` carries the reference ``cli.Task`` attributes the header needs (two_js, two_j12, two_j43, delta_12,
delta_43, delta_1_plus_2, q4, sign, order, Lambda, kept_pole_order, coordinates, precision,
two_js_internal, out_template, argv).  ``device_outputs[coord]`` is the drop-in's MPF (Jo, 2, S^2, nq,
outputs, Dmax) on the GPU (``dropin.Operator.apply_outputs``).

Work per file set: one formatting kernel over every number (``b3d_format_decimal``), one kernel for the
kept sizes and text lengths of every polynomial (``b3d_poly_sizes``), a prefix sum of the lengths and one
assembly kernel (``b3d_emit_text``) that writes header, brackets and numbers of all files into one device
buffer; one device-to-host copy brings the files back.  The header and the bracket "skeleton" are built
on the host once per (task, shapes) and cached.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib, structure as S
from .mpf import MPF

COORD_ORDER = ["zzb", "yyb", "xt", "ws", "xt_radial", "ws_radial"]      # blocks_3d's std::set<Coordinate> order


def digits10(precision):
    """digits of blocks_3d's output at an input precision in bits (``b3djson.py:20-23``)"""
    return ((precision - 1) // 64 + 1) * 64 * 301 // 1000


def precision_actual(p):
    return int((p + 1) * math.log(10.0) / math.log(2.0))


def eps_shift(p):
    """blocks_3d's truncation threshold eps = 2^-eps_shift(p) (``b3djson.py:176-179``)"""
    return 1 + int(0.9 * math.log2(10) * p)


def slot_stride(p):
    return (p + 12 + 15) // 16 * 16


def _limbs_of(v, n):
    return np.frombuffer(int(v).to_bytes(4 * n, "little"), dtype="<u4")


class _Tables:
    """device tables of the formatter for (L, p): 5^k for k <= 3p, 10^(p-1) and 10^p"""

    def __init__(self, L, p, device):
        kmax = 3 * p
        fw = (5 ** kmax).bit_length() // 32 + 1
        pow5 = np.zeros((kmax + 1, fw), dtype=np.uint32)
        nl = np.zeros(kmax + 1, dtype=np.int32)
        v = 1
        for k in range(kmax + 1):
            pow5[k] = _limbs_of(v, fw)
            nl[k] = (v.bit_length() + 31) // 32
            v *= 5
        bounds = np.stack([_limbs_of(10 ** (p - 1), L - 1), _limbs_of(10 ** p, L - 1)])
        self.pow5 = torch.from_numpy(pow5.view(np.int32)).to(device)
        self.nl = torch.from_numpy(nl).to(device)
        self.bounds = torch.from_numpy(bounds.view(np.int32).copy()).to(device)
        self.c = _lib.DecimalTables(self.pow5.data_ptr(), self.nl.data_ptr(), self.bounds.data_ptr(), kmax, fw, p,
                                    slot_stride(p))
        self.err = torch.zeros(2, dtype=torch.int64, device=device)


_TABLES = {}


def tables(L, p, device):
    key = (L, p, str(torch.device(device)))
    if key not in _TABLES:
        _TABLES[key] = _Tables(L, p, device)
    return _TABLES[key]


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def format_numbers(x, p, out=None, lens=None, check=True):
    """every number of the MPF x printed at p digits: (slots uint8 (n, stride), lengths int32 (n)).
    out / lens: preallocated buffers (n * stride bytes, 16-byte aligned; n int32)."""
    L, dev = x.L, x.m.device
    m = x.m.reshape(L, -1)
    e = x.e.reshape(-1)
    n = e.numel()
    tb = tables(L, p, dev)
    st = tb.c.stride
    out = torch.empty(n * st, dtype=torch.uint8, device=dev) if out is None else out
    lens = torch.empty(n, dtype=torch.int32, device=dev) if lens is None else lens
    tb.err[0], tb.err[1] = 0, (1 << 63) - 1
    _lib.call("b3d_format_decimal", L, m.data_ptr(), e.data_ptr(), m.stride(0), n, ctypes.byref(tb.c),
              out.data_ptr(), lens.data_ptr(), tb.err.data_ptr(), _stream(dev))
    if check:
        check_errors(L, p, dev)
    return out.view(n, st), lens


def check_errors(L, p, device):
    """raise if numbers fell outside the formatter's decimal range"""
    bad, first = (int(v) for v in tables(L, p, device).err.cpu())
    if bad:
        raise _lib.B3DError(f"b3d_format_decimal: {bad} numbers outside the supported decimal range "
                            f"(first at index {first})")


# ---------------------------------------------------------------- header (b3djson.header, b3djson.py:97-147)
def fmt_double(x, p):
    """std::ostream << double at precision p (general format)"""
    s = f"{float(x):.{p}g}"
    if "e" in s:
        mnt, ex = s.split("e")
        s = mnt + "e" + ex[0] + ex[1:].lstrip("0").rjust(2, "0")
    return s


def _fmt_half(a):
    """the printed form of the half-integer a / 2 (any p > the few digits it has)"""
    s = "-" if a < 0 else ""
    a = abs(a)
    return s + str(a // 2) + (".5" if a % 2 else "")


def _list(xs):
    return "[" + ", ".join(xs) + "]"


def header(o, two_j, pp, p):
    tjs, tj12, tj43 = o.two_js, o.two_j12, o.two_j43
    dbl = lambda x: fmt_double(x, p)
    ub2 = two_j + 1 if two_j <= 1 else two_j + 2                       # 2 x (Delta - x) bound
    ub = ub2 / 2.0
    poles = sorted({S.twice_position(P, two_j) - ub2 for P in S.block_poles(two_j, tj12, tj43, o.kept_pole_order)})
    coords = [c for c in COORD_ORDER if c in o.coordinates]
    out = ["{\n",
           f"  \"j_external\": {_list([dbl(x / 2.0) for x in tjs])},\n",
           f"  \"j_internal\": {dbl(two_j / 2.0)},\n",
           f"  \"delta_minus_x\": {dbl(ub)},\n",
           f"  \"j_12\": {dbl(tj12 / 2.0)},\n",
           f"  \"j_43\": {dbl(tj43 / 2.0)},\n",
           f"  \"delta_12\": \"{o.delta_12}\",\n",
           f"  \"delta_43\": \"{o.delta_43}\",\n",
           f"  \"delta_1_plus_2\": \"{o.delta_1_plus_2}\",\n",
           f"  \"four_pt_struct\": {_list([dbl(x / 2.0) for x in o.q4])},\n",
           f"  \"four_pt_sign\": {o.sign},\n",
           f"  \"order\": {o.order},\n",
           f"  \"lambda\": {o.Lambda},\n",
           f"  \"kept_pole_order\": {o.kept_pole_order},\n",
           "  \"coordinates\": [" + ",".join(f"\"{c}\"" for c in coords) + "],\n",
           "  \"pole_list_x\": [" + ", ".join(_fmt_half(a) for a in poles) + "],\n",
           f"  \"precision_input\": {o.precision},\n",
           f"  \"precision_actual\": {precision_actual(p)},\n",
           "  \"j_internal_input\": [" + ", ".join(dbl(x / 2.0) for x in o.two_js_internal) + "],\n",
           f"  \"output_template\": \"{o.out_template}\",\n",
           f"  \"args\": \"{' '.join(o.argv)}\",\n",
           "  \"index_values\": [\n"]
    for k in range(2):
        if k:
            out.append(",\n")
        par120 = abs((tj12 - tjs[0] + tjs[1]) // 2 + pp[k][0]) % 2
        par430 = abs((tj43 - tjs[3] + tjs[2]) // 2 + pp[k][1]) % 2
        out += ["    {\n",
                f"     \"three_pt_parity_120\": {par120},\n",
                f"     \"three_pt_parity_430\": {par430},\n",
                f"     \"j_120\": {_list([dbl(x / 2.0) for x in S.so3_structures(pp[k][0], tj12, two_j)])},\n",
                f"     \"j_430\": {_list([dbl(x / 2.0) for x in S.so3_structures(pp[k][1], tj43, two_j)])},\n",
                "     \"coordinates\": [" + ", ".join(f"\"{c}\"" for c in coords) + "]\n",
                "    }"]
    out.append("\n  ],\n")
    out.append("  \"index_names\": [\"three_pt_parity_index\",\n"
               "                  \"j_120_index\",\n"
               "                  \"j_430_index\",\n"
               "                  \"coordinate_index\",\n"
               "                  \"deriv_0\",\n"
               "                  \"deriv_1\",\n"
               "                  \"monomial_degree\"],\n")
    return "".join(out)


# ---------------------------------------------------------------- skeleton and device assembly
class _Skeleton:
    """the bytes between polynomials of every file of one task, and each polynomial's first number"""

    def __init__(self):
        self.pieces, self.polys, self.cur, self.file_first = [], [], [], []

    def text(self, s):
        self.cur.append(s)

    def poly(self, first):
        self.pieces.append("".join(self.cur))
        self.polys.append(first)
        self.cur = []

    def end_file(self):
        self.pieces.append("".join(self.cur))
        self.polys.append(-1)                                           # sentinel: skeleton only
        self.cur = []


class SpinWriter:
    """All spin files of one task (one right-hand-side column q of the drop-in's output arrays).
    outputs: {coord: Output.outputs list}; Smax, nq, Dmax: the output arrays' shape."""

    def __init__(self, opts, tjs, pp, outputs, Smax, nq, Dmax, device="cuda"):
        self.o, self.tjs, self.pp, self.Sm, self.nq, self.Dmax = opts, list(tjs), pp, Smax, nq, Dmax
        self.device = torch.device(device)
        self.p = digits10(opts.precision)
        self.coords = [c for c in COORD_ORDER if c in opts.coordinates]
        self.outputs = {c: list(outputs[c]) for c in self.coords}
        self._built = {}

    def _build(self, q, order):
        """skeleton + polynomial table for task column q; number indices are into the concatenation of the
        coordinates' arrays in `order` (each (Jo, 2, S^2, nq, outputs, Dmax))"""
        Sm2, nq, D = self.Sm * self.Sm, self.nq, self.Dmax
        Jo = len(self.tjs)
        base, off = {}, 0
        for c in order:
            base[c] = off
            off += Jo * 2 * Sm2 * nq * len(self.outputs[c]) * D
        rows_of = {}
        for c in self.coords:
            by_n = {}
            for idx, (n, _) in enumerate(self.outputs[c]):
                by_n.setdefault(n, []).append(idx)
            rows_of[c] = [by_n[n] for n in sorted(by_n)]
        sk = _Skeleton()
        files = []
        for tj in self.o.two_js_internal:
            jo = self.tjs.index(tj)
            files.append(tj)
            structs = [(len(S.so3_structures(self.pp[k][0], self.o.two_j12, tj)),
                        len(S.so3_structures(self.pp[k][1], self.o.two_j43, tj))) for k in range(2)]
            sk.text(header(self.o, tj, self.pp, self.p))
            sk.text("  \"derivs\":\n  [\n")
            for k in range(2):
                sk.text("    [\n")
                nl, nr = structs[k]
                for a in range(nl):
                    sk.text("      [\n")
                    for b in range(nr):
                        sk.text("        [\n")
                        for ci, c in enumerate(self.coords):
                            if ci:
                                sk.text(",\n")
                            nout = len(self.outputs[c])
                            cell = ((jo * 2 + k) * Sm2 + a * self.Sm + b) * nq + q
                            sk.text("          [\n")
                            rows = rows_of[c]
                            for d0, row in enumerate(rows):
                                sk.text("            [\n")
                                for d1, oi in enumerate(row):
                                    sk.text("              [\n")
                                    sk.poly(base[c] + (cell * nout + oi) * D)
                                    sk.text("\n              ]")
                                    if d1 + 1 != len(row):
                                        sk.text(",\n")
                                sk.text("\n            ]")
                                if d0 + 1 != len(rows):
                                    sk.text(",\n")
                            sk.text("\n          ]")
                        sk.text("\n        ]")
                        if b + 1 != nr:
                            sk.text(",\n")
                    sk.text("\n      ]")
                    if a + 1 != nl:
                        sk.text(",\n")
                sk.text("\n    ]")
                if k + 1 != 2:
                    sk.text(",\n")
            sk.text("\n  ]\n}\n")
            sk.end_file()
        blob = "".join(sk.pieces).encode()
        skel_off = np.zeros(len(sk.pieces) + 1, dtype=np.int64)
        skel_off[1:] = np.cumsum([len(s.encode()) for s in sk.pieces])
        polys = np.asarray(sk.polys, dtype=np.int64)
        dev = self.device
        ends = np.flatnonzero(polys < 0)                               # the sentinel of each file
        return dict(
            skel=torch.frombuffer(bytearray(blob), dtype=torch.uint8).to(dev) if blob else
            torch.zeros(1, dtype=torch.uint8, device=dev),
            skel_off=torch.from_numpy(skel_off).to(dev),
            skel_len=torch.from_numpy(np.diff(skel_off)).to(dev),
            poly_num=torch.from_numpy(np.where(polys < 0, 0, polys)).to(dev),
            sentinel=torch.from_numpy(polys < 0).to(dev),
            ends_dev=torch.from_numpy(ends).to(dev), files=files, npoly=len(polys))

    def render_device(self, outs, q=0, events=None):
        """every file of column q assembled on the GPU: (uint8 device buffer, [file end offsets], [two_j]).
        events: a list that receives (name, start, end) CUDA events around each kernel"""
        order = list(self.coords)
        key = (q, tuple(order))
        if key not in self._built:
            self._built[key] = self._build(q, order)
        b = self._built[key]
        if len(order) == 1:
            x = outs[order[0]]
        else:
            L = outs[order[0]].L
            x = MPF(torch.cat([outs[c].m.reshape(L, -1) for c in order], 1),
                    torch.cat([outs[c].e.reshape(-1) for c in order]))
        L, p, dev = x.L, self.p, self.device
        st = _stream(dev)

        def timed(name, fn):
            if events is None:
                return fn()
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
            r = fn()
            ev[1].record()
            events.append((name, ev[0], ev[1]))
            return r

        slots, lens = timed("b3d_format_decimal", lambda: format_numbers(x, p, check=False))
        m, e = x.m.reshape(L, -1), x.e.reshape(-1)
        npoly = b["npoly"]
        size = torch.empty(npoly, dtype=torch.int32, device=dev)
        tlen = torch.empty(npoly, dtype=torch.int64, device=dev)
        timed("b3d_poly_sizes", lambda: _lib.call(
            "b3d_poly_sizes", L, m.data_ptr(), e.data_ptr(), m.stride(0), b["poly_num"].data_ptr(), npoly, self.Dmax,
            eps_shift(p), lens.data_ptr(), size.data_ptr(), tlen.data_ptr(), st))
        size.masked_fill_(b["sentinel"], -1)
        tlen.masked_fill_(b["sentinel"], 0)
        nbad = int((tlen < 0).sum())
        if nbad:
            raise _lib.B3DError(f"JSON output: {nbad} polynomials keep a coefficient outside the decimal "
                                f"formatter's range")
        tot = b["skel_len"] + tlen
        ends = torch.cumsum(tot, 0)
        out_off = ends - tot
        total = int(ends[-1])
        out = torch.empty(total, dtype=torch.uint8, device=dev)
        timed("b3d_emit_text", lambda: _lib.call(
            "b3d_emit_text", slots.data_ptr(), slots.shape[1], lens.data_ptr(), b["poly_num"].data_ptr(),
            size.data_ptr(), out_off.data_ptr(), b["skel"].data_ptr(), b["skel_off"].data_ptr(), npoly,
            out.data_ptr(), st))
        file_ends = [int(v) for v in ends[b["ends_dev"]].cpu()]
        self.last_numbers = e.numel()
        return out, file_ends, b["files"]

    def render(self, outs, q=0):
        """outs: {coord: MPF (Jo, 2, S^2, nq, outputs, Dmax) on the GPU}.  Returns {two_j: file bytes} as
        memoryviews of one pinned host buffer (no host-side copies), valid until the next render."""
        out, ends, files = self.render_device(outs, q)
        n = out.numel()
        if getattr(self, "_pinned", None) is None or self._pinned.numel() < n:
            self._pinned = torch.empty(max(n, 1), dtype=torch.uint8, pin_memory=True)
        host = self._pinned[:n]
        host.copy_(out)
        mv = memoryview(host.numpy())
        bounds = [0] + ends
        return {tj: mv[bounds[i]:bounds[i + 1]] for i, tj in enumerate(files)}

    def write(self, outs, path_of, q=0):
        """render and write every file: path_of(two_j) -> path (the reference's Task.path(j))"""
        import os
        for tj, view in self.render(outs, q).items():
            path = path_of(tj)
            os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
            with open(path, "wb") as f:
                f.write(view)


def task_options(group, task, out_template="out/block_{}.json", argv=()):
    """the reference cli.Task attributes the file header reads, from a drop-in group and task"""
    from types import SimpleNamespace
    return SimpleNamespace(two_js=tuple(group.two_js), two_j12=group.two_j12, two_j43=group.two_j43,
                           delta_12=group.delta_12, delta_43=group.delta_43, delta_1_plus_2=task.delta_1_plus_2,
                           q4=tuple(task.q4), sign=task.sign, order=group.order, Lambda=group.Lambda,
                           kept_pole_order=group.kept_pole_order, coordinates=tuple(task.coordinates),
                           precision=group.precision, two_js_internal=list(task.two_js_internal),
                           out_template=out_template, argv=list(argv))
