"""Generate the CO2-Ar PES and induced-dipole coefficient tables.

The CO2-Ar surfaces of HAWAIIHYBRID are Maple-generated piecewise functions of
(R, theta) in the molecular frame (``PES-IDS/ai_pes_co2ar.c:27-459`` for the
potential, ``PES-IDS/ai_ids_co2ar.cpp:21-491`` for the two body-frame dipole
components).  Each R-interval is a sum over Legendre functions P_l^m(cos theta)
(l = 0, 2, ..., 10; m = 0 for V and d_z, m = 1 for d_x) times a radial function
of R: a cubic polynomial, an exponential (R < 4.5 in V) or inverse powers of R
(R >= 20 in the dipole, R >= 30 in V).

This script parses those expressions with exact rational arithmetic
(``fractions.Fraction`` of the decimal literals), collects for every interval and
every (l, m) the radial function, re-centres each polynomial part on the
interval start (c(R) = sum_k a_k (R - R_lo)^k, which removes the cancellation of
the monomial form and keeps FP32 evaluation well conditioned) and writes one
C header of ``static const double`` tables that both the CUDA kernels and the
CPU oracle include.  The numbers are the reference's fit coefficients; only
their arrangement is new.

Usage: python gen_co2ar_tables.py <reference root> <output header>
"""
from __future__ import annotations

import re
import sys
from fractions import Fraction
from math import comb

NL = 6                      # l = 0, 2, 4, 6, 8, 10
NPOLY = 4                   # cubic in (R - R_lo)
INV_POWERS = (4, 5, 6, 7)   # R^-4 .. R^-7 terms


class Expr:
    """Sum of terms keyed by (l, m, kind, k, p) with exact coefficients.

    kind 'p': coeff * R^p * P_l^m            (p may be negative)
    kind 'e': coeff * exp(k R) * R^p * P_l^m
    The key (l, m) = (-1, -1) marks a term without a Legendre factor.
    """

    def __init__(self, terms=None):
        self.t = dict(terms or {})

    @staticmethod
    def const(c):
        return Expr({(-1, -1, 'p', Fraction(0), 0): Fraction(c)})

    @staticmethod
    def R():
        return Expr({(-1, -1, 'p', Fraction(0), 1): Fraction(1)})

    @staticmethod
    def leg(l, m):
        return Expr({(l, m, 'p', Fraction(0), 0): Fraction(1)})

    @staticmethod
    def expo(arg: "Expr"):
        # arg must be k*R
        assert len(arg.t) == 1, arg.t
        (key, c), = arg.t.items()
        assert key[0] == -1 and key[2] == 'p' and key[4] == 1, key
        return Expr({(-1, -1, 'e', c, 0): Fraction(1)})

    def _lift(self, o):
        if isinstance(o, Expr):
            return o
        return Expr.const(o)

    def __add__(self, o):
        o = self._lift(o)
        r = dict(self.t)
        for k, v in o.t.items():
            r[k] = r.get(k, 0) + v
        return Expr(r)

    __radd__ = __add__

    def __neg__(self):
        return Expr({k: -v for k, v in self.t.items()})

    def __sub__(self, o):
        return self + (-self._lift(o))

    def __rsub__(self, o):
        return self._lift(o) - self

    def __mul__(self, o):
        o = self._lift(o)
        r = {}
        for (l1, m1, k1, e1, p1), c1 in self.t.items():
            for (l2, m2, k2, e2, p2), c2 in o.t.items():
                if l1 >= 0 and l2 >= 0:
                    raise ValueError("product of two Legendre factors")
                l, m = (l1, m1) if l1 >= 0 else (l2, m2)
                if k1 == 'e' and k2 == 'e':
                    raise ValueError("product of two exponentials")
                kind = 'e' if 'e' in (k1, k2) else 'p'
                e = e1 if k1 == 'e' else e2
                key = (l, m, kind, e, p1 + p2)
                r[key] = r.get(key, 0) + c1 * c2
        return Expr(r)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = self._lift(o)
        assert len(o.t) == 1, "division only by a monomial"
        (key, c), = o.t.items()
        assert key[0] == -1 and key[2] == 'p', key
        inv = Expr({(-1, -1, 'p', Fraction(0), -key[4]): 1 / c})
        return self * inv

    def __rtruediv__(self, o):
        return self._lift(o) * (Expr.const(1) / self)


NUM = re.compile(r'(?<![\w.])(\d+\.\d*(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)')


def to_python(expr: str) -> str:
    expr = expr.replace('std::', '')
    expr = re.sub(r'LegP\[index\((\d+),\s*(\d+)\)\]', r'_leg(\1,\2)', expr)
    expr = re.sub(r'legP\[(\d+)\]', r'_leg(\1,0)', expr)
    expr = NUM.sub(lambda mt: f"_F('{mt.group(1)}')", expr)
    return expr


def strip_comments(src: str) -> str:
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return re.sub(r'//[^\n]*', '', src)


def parse_branches(src: str, fname: str):
    """Return [(upper_bound or None, {var: Expr}, result_var)] for one function."""
    src = strip_comments(src)
    start = re.search(fname, src).start()
    body_start = src.index('{', start)
    depth, i = 0, body_start
    while True:
        if src[i] == '{':
            depth += 1
        elif src[i] == '}':
            depth -= 1
            if depth == 0:
                break
        i += 1
    body = src[body_start + 1:i]
    # split on if / else if / else blocks
    pieces = re.split(r'\n\s*(?:else\s+)?if\s*\(R\s*<\s*([0-9.]+)\)\s*\n|\n\s*else\s*\n', body)
    # re.split with a capture group interleaves bounds; the final else has None
    out = []
    head = pieces[0]
    rest = pieces[1:]
    j = 0
    bounds = []
    blocks = []
    while j < len(rest):
        b = rest[j]
        blk = rest[j + 1]
        bounds.append(float(b) if b is not None else None)
        blocks.append(blk)
        j += 2
    for ub, blk in zip(bounds, blocks):
        env = {'_F': Fraction, '_leg': Expr.leg, 'exp': Expr.expo, 'R': Expr.R()}
        result = None
        for stmt in blk.split(';'):
            stmt = stmt.strip().strip('{}').strip()
            if not stmt or stmt.startswith('//') or stmt.startswith('(void)'):
                continue
            if stmt.startswith('return'):
                result = stmt.split()[1]
                continue
            if '=' not in stmt:
                continue
            lhs, rhs = stmt.split('=', 1)
            lhs = lhs.strip().split()[-1]
            env[lhs] = eval(to_python(' '.join(rhs.split())), {}, env)
        out.append((ub, env, result))
    return out


def collect(branches, result_var_default, scale=Fraction(1)):
    """Per interval: dict (l, m) -> {('p', p): c, ('e', k, p): c}."""
    intervals = []
    for ub, env, res in branches:
        var = res or result_var_default
        e = env[var]
        radial = {}
        for (l, m, kind, k, p), c in e.t.items():
            if c == 0:
                continue
            lm = (0, 0) if l < 0 else (l, m)
            key = ('p', p) if kind == 'p' else ('e', k, p)
            radial.setdefault(lm, {})
            radial[lm][key] = radial[lm].get(key, 0) + c * scale
        intervals.append((ub, radial))
    return intervals


def shift_poly(coeffs: dict, r0: Fraction):
    """Monomial powers 0..3 -> coefficients of (R - r0)^j."""
    out = [Fraction(0)] * NPOLY
    for p, a in coeffs.items():
        for j in range(p + 1):
            out[j] += a * comb(p, j) * r0 ** (p - j)
    return out


def build_table(intervals, lm_list, lower0):
    """Arrange into rows: [a0..a3 | b4..b7 | A, k]  per (interval, lm)."""
    rows = []
    bounds = []
    lo = Fraction(lower0)
    for ub, radial in intervals:
        bounds.append(float(ub) if ub is not None else float('inf'))
        r_lo = lo
        per_lm = []
        for lm in lm_list:
            d = radial.get(lm, {})
            poly = {}
            inv = {q: Fraction(0) for q in INV_POWERS}
            A = Fraction(0)
            kexp = Fraction(0)
            for key, c in d.items():
                if key[0] == 'p':
                    p = key[1]
                    if 0 <= p <= 3:
                        poly[p] = poly.get(p, 0) + c
                    elif -p in INV_POWERS:
                        inv[-p] += c
                    else:
                        raise ValueError(f"unsupported power {p} in interval < {ub}")
                else:
                    _, k, p = key
                    if p != 0:
                        raise ValueError("exp term with a polynomial factor")
                    if A != 0 and k != kexp:
                        raise ValueError("two exponentials for one (l, m)")
                    A += c
                    kexp = k
            a = shift_poly(poly, r_lo) if poly else [Fraction(0)] * NPOLY
            per_lm.append([float(x) for x in a] + [float(inv[q]) for q in INV_POWERS]
                          + [float(A), float(kexp)])
        rows.append((float(r_lo), per_lm))
        if ub is not None:
            lo = Fraction(str(ub))
    return rows


def emit(name, rows, fh):
    fh.write(f"/* {name}: [interval][l index][a0 a1 a2 a3 | b4 b5 b6 b7 | A k] */\n")
    fh.write(f"static const double {name}[{len(rows)}][{NL}][10] = {{\n")
    for r_lo, per_lm in rows:
        fh.write(f"  {{ /* R_lo = {r_lo!r} */\n")
        for row in per_lm:
            fh.write("    {" + ", ".join(repr(x) if x != 0 else "0.0" for x in row) + "},\n")
        fh.write("  },\n")
    fh.write("};\n")


def main():
    ref, out = sys.argv[1], sys.argv[2]
    pes_src = open(f"{ref}/PES-IDS/ai_pes_co2ar.c").read()
    ids_src = open(f"{ref}/PES-IDS/ai_ids_co2ar.cpp").read()

    # Potential in cm^-1 (the reference divides by HTOCM at return; the kernels do the same).
    pes = collect(parse_branches(pes_src, r'double\s+pes_co2ar\s*\(double R, double Theta\)\s*\{'), 't48')
    dipx = collect(parse_branches(ids_src, r'double\s+AI_IDS_co2_ar::dipx\s*\('), None)
    dipz = collect(parse_branches(ids_src, r'double\s+AI_IDS_co2_ar::dipz\s*\('), None)

    ls = [0, 2, 4, 6, 8, 10]
    bounds = [b for b, _ in pes]
    assert [b for b, _ in dipx] == bounds and [b for b, _ in dipz] == bounds

    pes_rows = build_table(pes, [(l, 0) for l in ls], 0)
    dx_rows = build_table(dipx, [(l, 1) for l in ls], 0)
    dz_rows = build_table(dipz, [(l, 0) for l in ls], 0)

    with open(out, 'w') as fh:
        fh.write("/* Generated by gen_co2ar_tables.py from the HAWAIIHYBRID CO2-Ar fits\n"
                 " * (PES-IDS/ai_pes_co2ar.c, PES-IDS/ai_ids_co2ar.cpp).  Do not edit. */\n")
        fh.write("#pragma once\n\n")
        fh.write(f"#define HH_CO2AR_NINT {len(bounds)}\n#define HH_CO2AR_NL {NL}\n\n")
        fh.write("/* upper bounds of the R intervals (bohr); the last one is open */\n")
        ub = [b for b in bounds[:-1]]
        fh.write(f"static const double hh_co2ar_rbound[{len(ub)}] = {{" + ", ".join(repr(b) for b in ub) + "};\n")
        fh.write(f"static const double hh_co2ar_rlo[{len(bounds)}] = {{" + ", ".join(repr(r) for r, _ in pes_rows) + "};\n\n")
        emit("hh_co2ar_pes", pes_rows, fh)
        emit("hh_co2ar_dipx", dx_rows, fh)
        emit("hh_co2ar_dipz", dz_rows, fh)


if __name__ == '__main__':
    main()
