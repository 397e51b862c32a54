"""Stand-ins for the reference's modules that are absent in this container (cupy, sdpvibe, gmpy2), so that its
CPU-side code (cli, b3djson, structure, the plan and output builders) imports and runs here.  Used only by the
fixture generators of tests/golden/ and by CPU tests that run the reference's own code when it is present.

gmpy2 is replaced by an exact mpmath-backed mpfr that supports what the reference's writer does with it
(b3djson.limbs_to_mpfr, write_spin(gmp=True), derivs_text): construction from ints, mul_2exp, abs, products,
comparisons, and "%.{p}g" formatting, which is delegated to the reference's own mpmath formatter fmt_big
(identical to MPFR's output except for values exactly halfway between two p-digit decimals)."""
import sys
import types

import mpmath as mp

EZ = -(1 << 60)


class _Mpfr:
    __slots__ = ("v",)

    def __init__(self, v=0):
        self.v = v.v if isinstance(v, _Mpfr) else mp.mpf(v)

    def __bool__(self):
        return bool(self.v)

    def __abs__(self):
        return _Mpfr(abs(self.v))

    def __neg__(self):
        return _Mpfr(-self.v)

    def _o(self, x):
        return x.v if isinstance(x, _Mpfr) else x

    def __mul__(self, x):
        return _Mpfr(self.v * self._o(x))

    __rmul__ = __mul__

    def __lt__(self, x):
        return self.v < self._o(x)

    def __gt__(self, x):
        return self.v > self._o(x)

    def __le__(self, x):
        return self.v <= self._o(x)

    def __ge__(self, x):
        return self.v >= self._o(x)

    def __eq__(self, x):
        return self.v == self._o(x)

    def __hash__(self):
        return hash(self.v)

    def __format__(self, spec):
        from blocksvibe import b3djson
        if not (spec.startswith(".") and spec.endswith("g")):
            raise ValueError(spec)
        return b3djson.fmt_big(self.v, int(spec[1:-1]))


def install(reference):
    """register the stand-ins and put the reference (its package and tests) on sys.path"""
    sys.path.insert(0, reference)
    for name in ("cupy", "sdpvibe", "sdpvibe.mpf", "sdpvibe.rns"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["sdpvibe"].mpf = sys.modules["sdpvibe.mpf"]
    sys.modules["sdpvibe"].rns = sys.modules["sdpvibe.rns"]
    sys.modules["sdpvibe.rns"].dev = "cpu"
    sys.modules["sdpvibe.mpf"].MPF = object
    sys.modules["sdpvibe.mpf"].EZ = EZ
    g = types.ModuleType("gmpy2")
    g.mpfr = _Mpfr
    g.mul_2exp = lambda x, k: _Mpfr(mp.ldexp(_Mpfr(x).v, int(k)))
    ctx = types.SimpleNamespace(precision=53)
    g.get_context = lambda: ctx
    sys.modules.setdefault("gmpy2", g)
    mp.mp.prec = max(mp.mp.prec, 4096)
