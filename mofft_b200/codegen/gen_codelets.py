"""CUDA radix-codelet generator: the sm_100a backend of the MoFFT kernel compiler.

The reference's build-time compiler (``compiler/mofft_compiler/emitter.py:283-466``
with the ``backends/arm_sme.py`` lowering) turns each radix-R DFT into SME
outer-product code.  On B200 a radix-R butterfly is a register-resident
straight-line program executed by one thread, so this generator emits, for
every radix the reference supports (``emitter.py:17``: 2..16, 32, 64), one
``__device__ __forceinline__`` function that computes, in place,

    y[k] = sum_j x[j] * exp(-2*pi*i*j*k/R)            (forward, FFTW sign)

which is the codelet contract of ``compiler/mofft_compiler/validate.py:115-127``
without the twiddle factor (twiddles are applied by the caller).  Backward
transforms use the identity  bwd(x) = conj(fwd(conj(x)))  in the kernels.

Algebra used (restated from the published methods, not from any library):
  * prime R: the conjugate-pair ("like terms") form of the reference's
    ``rewrites.py:43-95`` LIKE_TERMS pattern:  a_j = x_j + x_{R-j},
    b_j = x_j - x_{R-j};  y_k = x_0 + sum a_j cos(2 pi jk/R) - i sum b_j sin(..).
  * composite R = A*B: one level of Cooley-Tukey decimation in time with
    compile-time twiddles; multiplications by 1, -1, +-i are folded and
    multiplications by (+-1 +- i)/sqrt(2) use two real multiplies.

Rewrite families.  Besides the default codelet above, every radix gets one
codelet per algebraic rewrite the reference's compiler defines for it
(``rewrites.py:15-41``: DIRECT and LIKE_TERMS for every radix, EVEN_ODD and
LIKE_TERMS_EVEN_ODD for even radices, VECTOR_REUSE and
LIKE_TERMS_VECTOR_REUSE for radices divisible by four), each a different
straight-line evaluation order of the same DFT:
  * direct:       y_k = sum_j x_j W^jk, one complex linear form per output;
  * like_terms:   conjugate pairs a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j}
                  (and the middle element of an even radix), outputs k and
                  R - k from the same two partial sums;
  * even_odd:     E_k (even j) and O_k (odd j) for k < R/2, then
                  y_k = E_k + O_k and y_{k+R/2} = E_k - O_k;
  * like_terms_even_odd: E_k and O_k each from conjugate pairs of one parity;
  * vector_reuse: for s < R/4, the sums S_r of x_j W^js over j = r mod 4 and
                  the four outputs y_{s + qR/4} = sum_r S_r (-i)^(rq), so the
                  coefficients of the first quarter are reused (a radix-4
                  butterfly on the partial sums);
  * like_terms_vector_reuse: the same with conjugate pairs in the residue
                  classes 0 and 2 (j and R - j fall in the same class there).
``DftFamily<R, F>`` selects one; ``BankDft<R, BANK>`` is the codelet kernel
bank BANK runs (0 default, 1 like_terms, 2 like_terms_even_odd where the
radix is even, 3 like_terms_vector_reuse where it is divisible by four; the
default codelet where the bank's family is not defined, and for radix 32 and
64 stages, whose matrix forms would not fit a thread's registers).

Run:  python -m mofft_b200.codegen.gen_codelets <out_dir>
It writes ``codelets.cuh`` (device code) and ``codelet_costs.h`` (real add /
multiply counts per radix, used by the host cost model).
"""
from __future__ import annotations

import json
import math
import sys
from dataclasses import dataclass
from decimal import Decimal, getcontext
from fractions import Fraction
from pathlib import Path

RADICES = (2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32, 64)

# Cooley-Tukey split (A = inner DFT length, B = outer) per composite radix.
SPLIT = {4: (2, 2), 6: (2, 3), 8: (2, 4), 9: (3, 3), 10: (2, 5), 12: (4, 3),
         14: (2, 7), 15: (3, 5), 16: (4, 4), 32: (4, 8), 64: (8, 8)}

SQRT_HALF = math.sqrt(0.5)

getcontext().prec = 60


def _pi() -> Decimal:
    """pi to 60 digits by Machin's formula (arctan series in Decimal)."""
    def arctan_inv(x: int) -> Decimal:
        total = term = Decimal(1) / x
        x2 = x * x
        n = 1
        sign = 1
        while True:
            term /= x2
            n += 2
            sign = -sign
            delta = term / n
            if delta == 0 or abs(delta) < Decimal(10) ** -70:
                break
            total += sign * delta
        return total
    return 4 * (4 * arctan_inv(5) - arctan_inv(239))


_PI = _pi()


def _sin_cos_small(x: Decimal) -> tuple[Decimal, Decimal]:
    """Taylor series for |x| <= pi/4."""
    s = Decimal(0)
    c = Decimal(0)
    term_s = x
    term_c = Decimal(1)
    n = 0
    while True:
        s += term_s
        c += term_c
        n += 1
        term_s = -term_s * x * x / ((2 * n) * (2 * n + 1))
        term_c = -term_c * x * x / ((2 * n - 1) * (2 * n))
        if abs(term_s) < Decimal(10) ** -65 and abs(term_c) < Decimal(10) ** -65:
            return s, c


def cis_turns(num: int, den: int) -> tuple[float, float]:
    """(cos, sin) of 2*pi*num/den, correctly rounded to double.

    The fraction is reduced exactly to an octant before the series, so
    values such as cos(2*pi/3) come out as exactly -0.5."""
    num %= den
    # angle = 2*pi*num/den; octant index = floor(8*num/den)
    eighths = Fraction(8 * num, den)
    octant = int(eighths)
    rest = eighths - octant            # in [0, 1): fraction of pi/4
    if octant % 2 == 1:
        rest = 1 - rest
        mirror = True
    else:
        mirror = False
    x = _PI / 4 * Decimal(rest.numerator) / Decimal(rest.denominator)
    s, c = _sin_cos_small(x)
    if mirror:
        s, c = c, s
    # (c, s) is now cos/sin of (octant-reduced) angle in [0, pi/4] or mirror.
    quadrant = octant // 2
    if quadrant == 0:
        cr, sr = c, s
    elif quadrant == 1:
        cr, sr = -s, c
    elif quadrant == 2:
        cr, sr = -c, -s
    else:
        cr, sr = s, -c
    return float(cr), float(sr)


def _lit(value: float) -> str:
    if abs(value) < 1e-300:
        return "T(0)"
    return f"T({value!r})"


class Emitter:
    """Builds straight-line SSA code over named real temporaries."""

    def __init__(self) -> None:
        self.lines: list[str] = []
        self.count = 0
        self.adds = 0
        self.muls = 0
        self.instr = 0

    def tmp(self, expr: str, adds: int = 0, muls: int = 0) -> str:
        name = f"t{self.count}"
        self.count += 1
        self.lines.append(f"  const T {name} = {expr};")
        self.adds += adds
        self.muls += muls
        # a product feeding a sum fuses into one FMA: a temporary of m
        # products and a sums costs max(a, m) instructions (a negation none)
        self.instr += max(adds, muls) if muls else adds
        return name

    def peak_live(self, outputs) -> int:
        """Peak number of live temporaries in program order; the outputs stay
        live to the end."""
        import re
        first, last = {}, {}
        for i, line in enumerate(self.lines):
            name, expr = line.split(" = ", 1)
            name = name.split()[-1]
            first[name] = i
            last.setdefault(name, i)
            for used in re.findall(r"\bt\d+\b", expr):
                last[used] = i
        end = len(self.lines)
        for y in outputs:
            for part in y:
                for used in re.findall(r"\bt\d+\b", part):
                    last[used] = end
        delta = [0] * (end + 2)
        for name, i in first.items():
            delta[i] += 1
            delta[last[name] + 1] -= 1
        peak = live = 0
        for d in delta:
            live += d
            peak = max(peak, live)
        return peak

    # complex helpers: values are (re, im) tuples of temporaries/expressions
    def add(self, a, b):
        return (self.tmp(f"{a[0]} + {b[0]}", 1), self.tmp(f"{a[1]} + {b[1]}", 1))

    def sub(self, a, b):
        return (self.tmp(f"{a[0]} - {b[0]}", 1), self.tmp(f"{a[1]} - {b[1]}", 1))

    def mul_unit(self, a, num: int, den: int):
        """Multiply by exp(2*pi*i*num/den), folding the easy cases."""
        c, s = cis_turns(num, den)
        eps = 1e-14
        if abs(c - 1) < eps and abs(s) < eps:
            return a
        if abs(c + 1) < eps and abs(s) < eps:
            return (self.tmp(f"-{a[0]}"), self.tmp(f"-{a[1]}"))
        if abs(c) < eps and abs(s - 1) < eps:   # * i
            return (self.tmp(f"-{a[1]}"), self.tmp(f"{a[0]}"))
        if abs(c) < eps and abs(s + 1) < eps:   # * -i
            return (self.tmp(f"{a[1]}"), self.tmp(f"-{a[0]}"))
        if abs(abs(c) - SQRT_HALF) < eps and abs(abs(s) - SQRT_HALF) < eps:
            # (c + i s) = h * (sc + i ss) with h = sqrt(1/2), sc, ss = +-1
            sc = "+" if c > 0 else "-"
            ss = "+" if s > 0 else "-"
            # re = h*(sc*ar - ss*ai), im = h*(ss*ar + sc*ai)
            re_inner = self.tmp(f"{sc}{a[0]} {'-' if ss == '+' else '+'} {a[1]}", 1)
            im_inner = self.tmp(f"{ss}{a[0]} {'+' if sc == '+' else '-'} {a[1]}", 1)
            h = _lit(SQRT_HALF)
            return (self.tmp(f"{h} * {re_inner}", 0, 1),
                    self.tmp(f"{h} * {im_inner}", 0, 1))
        cl, sl = _lit(c), _lit(s)
        return (self.tmp(f"{a[0]} * {cl} - {a[1]} * {sl}", 1, 2),
                self.tmp(f"{a[0]} * {sl} + {a[1]} * {cl}", 1, 2))

    def dft(self, xs):
        radix = len(xs)
        if radix == 1:
            return list(xs)
        if radix == 2:
            return [self.add(xs[0], xs[1]), self.sub(xs[0], xs[1])]
        if radix in SPLIT:
            return self._cooley_tukey(xs, *SPLIT[radix])
        return self._prime(xs)

    def _prime(self, xs):
        radix = len(xs)
        half = (radix - 1) // 2
        a = [None] * (half + 1)
        b = [None] * (half + 1)
        for j in range(1, half + 1):
            a[j] = self.add(xs[j], xs[radix - j])
            b[j] = self.sub(xs[j], xs[radix - j])
        ys = [None] * radix
        acc = xs[0]
        for j in range(1, half + 1):
            acc = self.add(acc, a[j])
        ys[0] = acc
        for k in range(1, half + 1):
            cr_terms = [xs[0][0]]
            ci_terms = [xs[0][1]]
            sr_terms = []
            si_terms = []
            for j in range(1, half + 1):
                cos_v, sin_v = cis_turns(j * k, radix)
                cj, sj = _lit(cos_v), _lit(sin_v)
                cr_terms.append(f"{a[j][0]} * {cj}")
                ci_terms.append(f"{a[j][1]} * {cj}")
                sr_terms.append(f"{b[j][0]} * {sj}")
                si_terms.append(f"{b[j][1]} * {sj}")
            n = len(sr_terms)
            cr = self.tmp(" + ".join(cr_terms), n, n)
            ci = self.tmp(" + ".join(ci_terms), n, n)
            sr = self.tmp(" + ".join(sr_terms), n - 1, n)
            si = self.tmp(" + ".join(si_terms), n - 1, n)
            ys[k] = (self.tmp(f"{cr} + {si}", 1), self.tmp(f"{ci} - {sr}", 1))
            ys[radix - k] = (self.tmp(f"{cr} - {si}", 1),
                             self.tmp(f"{ci} + {sr}", 1))
        return ys

    def _cooley_tukey(self, xs, inner: int, outer: int):
        radix = inner * outer
        z = []
        for n2 in range(outer):
            col = self.dft([xs[outer * n1 + n2] for n1 in range(inner)])
            z.append([self.mul_unit(col[k1], -n2 * k1, radix)
                      for k1 in range(inner)])
        ys = [None] * radix
        for k1 in range(inner):
            row = self.dft([z[n2][k1] for n2 in range(outer)])
            for k2 in range(outer):
                ys[k1 + inner * k2] = row[k2]
        return ys


    # ---------------------------------------------------------- families
    def linear(self, xs, coeffs):
        """sum_j coeffs[j] * xs[j] for compile-time complex coefficients
        (real, imaginary) pairs; zero and unit parts fold away."""
        eps = 1e-14
        re_terms, im_terms = [], []
        muls = 0
        for x, (c, s) in zip(xs, coeffs):
            # c * (xr + i xi) contributes (c xr, c xi); i s * x gives (-s xi, s xr)
            for coef, part_re, part_im in ((c, x[0], x[1]), (s, f"-{x[1]}", x[0])):
                if abs(coef) < eps:
                    continue
                if abs(coef - 1) < eps:
                    re_terms.append(part_re)
                    im_terms.append(part_im)
                elif abs(coef + 1) < eps:
                    re_terms.append(f"-({part_re})")
                    im_terms.append(f"-({part_im})")
                else:
                    lit = _lit(coef)
                    re_terms.append(f"({part_re}) * {lit}")
                    im_terms.append(f"({part_im}) * {lit}")
                    muls += 2
        if not re_terms:
            return (self.tmp("T(0)"), self.tmp("T(0)"))
        adds = len(re_terms) - 1
        return (self.tmp(" + ".join(re_terms), adds, muls // 2),
                self.tmp(" + ".join(im_terms), adds, muls - muls // 2))

    def _w(self, j: int, k: int, radix: int):
        """Forward coefficient W^jk = cos - i sin of 2 pi jk / R."""
        c, s = cis_turns(j * k, radix)
        return (c, -s)

    def family(self, xs, fam: str):
        radix = len(xs)
        if fam == "direct":
            return [self.linear(xs, [self._w(j, k, radix) for j in range(radix)])
                    for k in range(radix)]
        if fam == "like_terms":
            return self._like_terms(xs)
        if fam in ("even_odd", "like_terms_even_odd"):
            half = radix // 2
            ys = [None] * radix
            if fam == "even_odd":
                evens = list(range(0, radix, 2))
                odds = list(range(1, radix, 2))
                for k in range(half):
                    e = self.linear([xs[j] for j in evens], [self._w(j, k, radix) for j in evens])
                    o = self.linear([xs[j] for j in odds], [self._w(j, k, radix) for j in odds])
                    ys[k] = self.add(e, o)
                    ys[k + half] = self.sub(e, o)
                return ys
            pairs = self._pairs(xs)
            for k in range(half):
                e = self._paired_sum(xs, pairs, k, parity=0)
                o = self._paired_sum(xs, pairs, k, parity=1)
                ys[k] = self.add(e, o)
                ys[k + half] = self.sub(e, o)
            return ys
        if fam in ("vector_reuse", "like_terms_vector_reuse"):
            q = radix // 4
            pairs = self._pairs(xs) if fam == "like_terms_vector_reuse" else None
            ys = [None] * radix
            for s_ in range(q):
                sums = []
                for r in range(4):
                    if pairs is not None and r in (0, 2):
                        sums.append(self._paired_sum(xs, pairs, s_, residue=r))
                    else:
                        js = [j for j in range(radix) if j % 4 == r]
                        sums.append(self.linear([xs[j] for j in js],
                                                [self._w(j, s_, radix) for j in js]))
                s0, s1, s2, s3 = sums
                a02, d02 = self.add(s0, s2), self.sub(s0, s2)
                a13, d13 = self.add(s1, s3), self.sub(s1, s3)
                mi = (self.tmp(f"{d13[1]}"), self.tmp(f"-{d13[0]}"))   # -i (s1 - s3)
                ys[s_] = self.add(a02, a13)
                ys[s_ + q] = self.add(d02, mi)
                ys[s_ + 2 * q] = self.sub(a02, a13)
                ys[s_ + 3 * q] = self.sub(d02, mi)
            return ys
        raise ValueError(fam)

    def _pairs(self, xs):
        """a_j = x_j + x_{R-j}, b_j = x_j - x_{R-j} for 1 <= j < R/2."""
        radix = len(xs)
        out = {}
        for j in range(1, (radix + 1) // 2):
            out[j] = (self.add(xs[j], xs[radix - j]), self.sub(xs[j], xs[radix - j]))
        return out

    def _paired_sum(self, xs, pairs, k, parity=None, residue=None):
        """sum over j of x_j W^jk (the pairs j, R-j together) restricted to
        j of one parity or one residue mod 4: x_j W^jk + x_{R-j} W^-jk =
        a_j cos - i b_j sin."""
        radix = len(xs)

        def keep(j):
            if parity is not None:
                return j % 2 == parity
            if residue is not None:
                return j % 4 == residue
            return True
        terms, coeffs = [], []
        if keep(0):
            terms.append(xs[0])
            coeffs.append((1.0, 0.0))
        if radix % 2 == 0 and keep(radix // 2):
            terms.append(xs[radix // 2])
            coeffs.append(self._w(radix // 2, k, radix))
        for j, (a, b) in pairs.items():
            if not keep(j):
                continue
            c, s = cis_turns(j * k, radix)
            terms.append(a)
            coeffs.append((c, 0.0))
            terms.append(b)
            coeffs.append((0.0, -s))
        return self.linear(terms, coeffs)

    def _like_terms(self, xs):
        radix = len(xs)
        pairs = self._pairs(xs)
        ys = [None] * radix
        ys[0] = self._paired_sum(xs, pairs, 0)
        for k in range(1, radix // 2 + 1):
            # C_k: x_0, middle and a_j cos; S_k: b_j sin.  y_k = C - i S,
            # y_{R-k} = C + i S
            cterms, ccoef = [xs[0]], [(1.0, 0.0)]
            if radix % 2 == 0:
                cterms.append(xs[radix // 2])
                ccoef.append(self._w(radix // 2, k, radix))
            sterms, scoef = [], []
            for j, (a, b) in pairs.items():
                c, s_ = cis_turns(j * k, radix)
                cterms.append(a)
                ccoef.append((c, 0.0))
                sterms.append(b)
                scoef.append((s_, 0.0))
            cc = self.linear(cterms, ccoef)
            ss = self.linear(sterms, scoef) if sterms else (self.tmp("T(0)"), self.tmp("T(0)"))
            if 2 * k == radix:
                ys[k] = cc
            else:
                ys[k] = (self.tmp(f"{cc[0]} + {ss[1]}", 1), self.tmp(f"{cc[1]} - {ss[0]}", 1))
                ys[radix - k] = (self.tmp(f"{cc[0]} - {ss[1]}", 1),
                                 self.tmp(f"{cc[1]} + {ss[0]}", 1))
        return ys


FAMILIES = ("direct", "like_terms", "even_odd", "like_terms_even_odd", "vector_reuse",
            "like_terms_vector_reuse")
FAMILY_ID = {name: i + 1 for i, name in enumerate(FAMILIES)}   # 0 = default codelet
BANK_COUNT = 4


def family_defined(radix: int, fam: str) -> bool:
    """rewrites.py:24-41: which rewrites are defined for a radix."""
    if fam in ("direct", "like_terms"):
        return True
    if fam in ("even_odd", "like_terms_even_odd"):
        return radix % 2 == 0
    return radix % 4 == 0


# ---------------------------------------------------------------- portfolio
# Candidates per radix (the counterpart of the reference compiler's candidate
# enumeration, compiler/mofft_compiler/patterns.py:607-628): every
# Cooley-Tukey split A x B of a composite radix (its sub-DFTs in their default
# form), the conjugate-pair form of a prime radix, the radix-2 butterfly, and
# every rewrite family defined for the radix (radices up to 16; larger ones
# would not fit a thread's registers in matrix form).  Ranked by a
# register-level cost model (model.py:293-323 ranks the reference's
# candidates with its SME model):
#   instructions  one per add, FMA-fused where a product feeds a sum;
#   registers     the peak number of live temporaries in program order; each
#                 value beyond REG_BUDGET costs SPILL_COST instructions (a
#                 spill store and reload);
#   cost          instructions + spill penalty; ties keep the default codelet
#                 first, then the name order.
# Banks (portfolio.py:31-35): bank 0 -- every specialised kernel -- runs the
# best-ranked candidate of every radix (ties keep the hand-chosen form: the
# split of SPLIT, the conjugate-pair form of a prime); bank B > 0 runs the
# best-ranked candidate carrying its family's rewrite (BANK_REWRITE:
# like-terms, even-odd, vector-reuse; the combined forms carry two), else
# bank 0's codelet.

REG_BUDGET = 64
SPILL_COST = 2
BANK_REWRITE = {1: "like_terms", 2: "even_odd", 3: "vector_reuse"}


@dataclass(frozen=True)
class Candidate:
    radix: int
    name: str            # "split_AxB", "prime", "radix2" or a family name
    family: str | None   # the rewrite family, None for the default forms
    adds: int
    muls: int
    instr: int
    live: int
    cost: int
    default: bool        # the hand-chosen form (SPLIT, prime, radix 2)


def _default_name(radix: int) -> str:
    if radix == 2:
        return "radix2"
    if radix in SPLIT:
        a, b = SPLIT[radix]
        return f"split_{a}x{b}"
    return "prime"


def _measure(radix: int, name: str, family: str | None) -> Candidate:
    em = Emitter()
    loaded = [(em.tmp(f"re[{j}]"), em.tmp(f"im[{j}]")) for j in range(radix)]
    if family is not None:
        ys = em.family(loaded, family)
    elif name.startswith("split_"):
        a, b = (int(v) for v in name[len("split_"):].split("x"))
        ys = em._cooley_tukey(loaded, a, b)
    else:
        ys = em.dft(loaded)
    live = em.peak_live(ys)
    cost = em.instr + SPILL_COST * max(0, live - REG_BUDGET)
    return Candidate(radix, name, family, em.adds, em.muls, em.instr, live, cost,
                     family is None and name == _default_name(radix))


def candidates(radix: int) -> list[Candidate]:
    """Every candidate codelet of a radix."""
    names: list[tuple[str, str | None]] = []
    if radix == 2:
        names.append(("radix2", None))
    elif any(radix % a == 0 for a in range(2, radix)):
        for a in range(2, radix):
            if radix % a == 0:
                names.append((f"split_{a}x{radix // a}", None))
    else:
        names.append(("prime", None))
    if radix <= 16:
        names += [(fam, fam) for fam in FAMILIES if family_defined(radix, fam)]
    return [_measure(radix, n, f) for n, f in names]


def ranked(radix: int) -> list[Candidate]:
    """Candidates of a radix, best first."""
    return sorted(candidates(radix), key=lambda c: (c.cost, not c.default, c.name))


def default_candidate(radix: int) -> Candidate:
    """The codelet bank 0 (every specialised kernel) runs for `radix`: the
    best-ranked candidate (ties keep the hand-chosen form)."""
    return ranked(radix)[0]


def bank_candidate(radix: int, bank: int) -> Candidate:
    """The codelet kernel bank `bank` runs for `radix`."""
    default = default_candidate(radix)
    if bank == 0:
        return default
    rewrite = BANK_REWRITE[bank]
    return next((c for c in ranked(radix) if c.family and rewrite in c.family), default)


def bank_family(radix: int, bank: int) -> str | None:
    """Rewrite family of bank `bank`'s codelet for `radix`; None where the
    bank runs the default codelet."""
    if bank == 0 or radix > 16:
        return None
    c = bank_candidate(radix, bank)
    return None if c == default_candidate(radix) else c.family


def portfolio_report() -> dict:
    """Every radix's ranked candidates and each bank's choice (JSON)."""
    out = {"reg_budget": REG_BUDGET, "spill_cost": SPILL_COST, "radices": {}}
    for radix in RADICES:
        out["radices"][str(radix)] = {
            "ranked": [{"name": c.name, "adds": c.adds, "muls": c.muls, "instr": c.instr,
                        "live": c.live, "cost": c.cost, "default": c.default}
                       for c in ranked(radix)],
            "banks": [bank_candidate(radix, b if radix <= 16 else 0).name
                      for b in range(BANK_COUNT)],
        }
    return out


def emit_family(radix: int, fam: str) -> str:
    em = Emitter()
    xs = [(f"re[{j}]", f"im[{j}]") for j in range(radix)]
    loaded = [(em.tmp(x[0]), em.tmp(x[1])) for x in xs]
    ys = em.family(loaded, fam)
    body = list(em.lines)
    for k, (yr, yi) in enumerate(ys):
        body.append(f"  re[{k}] = {yr};")
        body.append(f"  im[{k}] = {yi};")
    return (f"template <typename T>\n"
            f"__device__ __forceinline__ void dft_fwd_{radix}_{fam}(T (&re)[{radix}], "
            f"T (&im)[{radix}]) {{\n" + "\n".join(body) + "\n}\n")


def emit_radix(radix: int) -> tuple[str, int, int]:
    """The default codelet of a radix: its best-ranked candidate."""
    em = Emitter()
    xs = []
    for j in range(radix):
        xs.append((f"re[{j}]", f"im[{j}]"))
    # Load inputs into named temporaries so writes to re/im cannot alias reads.
    loaded = [(em.tmp(x[0]), em.tmp(x[1])) for x in xs]
    best = default_candidate(radix)
    if best.family is not None:
        ys = em.family(loaded, best.family)
    elif best.name.startswith("split_") and best.name != _default_name(radix):
        a, b = (int(v) for v in best.name[len("split_"):].split("x"))
        ys = em._cooley_tukey(loaded, a, b)
    else:
        ys = em.dft(loaded)
    body = list(em.lines)
    for k, (yr, yi) in enumerate(ys):
        body.append(f"  re[{k}] = {yr};")
        body.append(f"  im[{k}] = {yi};")
    text = (f"template <typename T>\n"
            f"__device__ __forceinline__ void dft_fwd_{radix}(T (&re)[{radix}], "
            f"T (&im)[{radix}]) {{\n" + "\n".join(body) + "\n}\n")
    return text, em.adds, em.muls


HEADER = """// Generated by mofft_b200/codegen/gen_codelets.py -- do not edit.
// Forward radix-R DFT codelets (FFTW sign), in place on register arrays.
#pragma once
"""


def generate() -> tuple[str, str]:
    parts = [HEADER]
    costs = []
    for radix in RADICES:
        text, adds, muls = emit_radix(radix)
        parts.append(text)
        default = bank_candidate(radix, 0)
        costs.append((radix, adds, muls, default.instr, default.live))
    dispatch = ["template <int R> struct Dft;"]
    for radix in RADICES:
        dispatch.append(
            f"template <> struct Dft<{radix}> {{ template <typename T> "
            f"__device__ __forceinline__ static void fwd(T (&re)[{radix}], "
            f"T (&im)[{radix}]) {{ dft_fwd_{radix}(re, im); }} }};")
    parts.append("\n".join(dispatch) + "\n")
    # rewrite families
    for radix in RADICES:
        for fam in FAMILIES:
            if family_defined(radix, fam):
                parts.append(emit_family(radix, fam))
    fam_lines = ["// Codelet of rewrite family F (1-based index into " +
                 ", ".join(FAMILIES) + ").",
                 "template <int R, int F> struct DftFamily;"]
    for radix in RADICES:
        for fam in FAMILIES:
            if family_defined(radix, fam):
                fam_lines.append(
                    f"template <> struct DftFamily<{radix}, {FAMILY_ID[fam]}> {{ "
                    f"template <typename T> __device__ __forceinline__ static void "
                    f"fwd(T (&re)[{radix}], T (&im)[{radix}]) {{ "
                    f"dft_fwd_{radix}_{fam}(re, im); }} }};")
    fam_lines.append("// Codelet kernel bank B runs for radix R (families for radices up to 16;")
    fam_lines.append("// radix-32 and -64 stages keep the split codelet in every bank).")
    fam_lines.append("template <int R, int B> struct BankDft : Dft<R> {};")
    for radix in (r for r in RADICES if r <= 16):
        for bank in range(1, BANK_COUNT):
            fam = bank_family(radix, bank)
            if fam is not None:
                fam_lines.append(
                    f"template <> struct BankDft<{radix}, {bank}> : "
                    f"DftFamily<{radix}, {FAMILY_ID[fam]}> {{}};")
    parts.append("\n".join(fam_lines) + "\n")
    cost_lines = [
        "// Generated by mofft_b200/codegen/gen_codelets.py -- do not edit.",
        "// Real additions / multiplications of one forward radix-R codelet (the",
        "// default form), its instructions with products fused into sums (FMA)",
        "// and its peak live temporaries.",
        "#pragma once",
        "typedef struct { int radix; int adds; int muls; int instr; int live; } "
        "mofft_codelet_cost;",
        "static const mofft_codelet_cost k_mofft_codelet_costs[] = {",
    ]
    for radix, adds, muls, instr, live in costs:
        cost_lines.append(f"  {{{radix}, {adds}, {muls}, {instr}, {live}}},")
    cost_lines.append("};")
    cost_lines.append(f"#define MOFFT_CODELET_COST_COUNT {len(costs)}")
    return "\n".join(parts), "\n".join(cost_lines) + "\n"


def main(argv: list[str]) -> int:
    out_dir = Path(argv[1]) if len(argv) > 1 else Path(__file__).resolve().parents[1] / "csrc" / "generated"
    out_dir.mkdir(parents=True, exist_ok=True)
    cuh, costs = generate()
    report = json.dumps(portfolio_report(), indent=1) + "\n"
    for name, text in (("codelets.cuh", cuh), ("codelet_costs.h", costs),
                       ("codelet_portfolio.json", report)):
        path = out_dir / name
        if not path.exists() or path.read_text() != text:
            path.write_text(text)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
