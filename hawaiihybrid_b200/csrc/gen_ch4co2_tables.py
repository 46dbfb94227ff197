#!/usr/bin/env python3
"""Generate hh_ch4co2_tables.h: the CH4-CO2 induced-dipole surface as data.

Reads PES-IDS/ai_ids_ch4_co2.cpp of a HAWAIIHYBRID source tree, whose
dipole_vector (ai_ids_ch4_co2.cpp:672-1067) is

    mu_c(R, phi1, theta1, phi2, theta2) = sum_b radcoeff_b(R) Re(idsbf_b(angles))_c

over 320 basis functions, and writes:

  * the radial functions: all 320 share one grid (a cubic piece below 5 bohr
    centred at 4.75, cubic pieces between the knots 5, 5.25, ..., 25, 30, and
    (quadratic in R) * R^-6 from 30 on).  Each piece is re-expanded exactly, in
    rational arithmetic, in powers of x = R - (its left knot) (4.75 for the first
    piece, 30 for the tail, whose value is then multiplied by R^-6);
  * the angular functions: every idsbf_b is expanded, exactly, into a sum of
    products  coef * P_l1^m1(cos theta1) trig(m1 phi1) * P_l2^m2(cos theta2) trig(m2 phi2)
    (GSL unnormalised associated Legendre functions with the Condon-Shortley
    phase, trig = cos or sin; the generator checks that the harmonic order of
    every trig factor equals the m of its Legendre factor).

A harmonic (l, m, cs) is stored as the integer  2 * (l(l+1)/2 + m) + cs  with cs = 0
for cos (and for m = 0, no trig factor) and cs = 1 for sin.

The script checks the expansion against a direct evaluation of the source's own
expressions at random points before it writes the header.

usage: gen_ch4co2_tables.py <reference-root> <output header>
"""
from __future__ import annotations

import ast
import math
import random
import re
import sys
from fractions import Fraction

SRC = "PES-IDS/ai_ids_ch4_co2.cpp"


# ----------------------------------------------------------------------------
# exact polynomial arithmetic: dict {monomial (sorted tuple of symbols): Fraction}
# ----------------------------------------------------------------------------
def p_add(a, b, s=1):
    r = dict(a)
    for k, v in b.items():
        r[k] = r.get(k, 0) + s * v
        if r[k] == 0:
            del r[k]
    return r


def p_mul(a, b):
    r = {}
    for ka, va in a.items():
        for kb, vb in b.items():
            k = tuple(sorted(ka + kb))
            r[k] = r.get(k, 0) + va * vb
    return {k: v for k, v in r.items() if v != 0}


def literal(node):
    return Fraction(ast.get_source_segment(literal.src, node))


def p_eval(node, env):
    if isinstance(node, ast.BinOp):
        a, b = p_eval(node.left, env), p_eval(node.right, env)
        if isinstance(node.op, ast.Add):
            return p_add(a, b)
        if isinstance(node.op, ast.Sub):
            return p_add(a, b, -1)
        if isinstance(node.op, ast.Mult):
            return p_mul(a, b)
        raise ValueError(ast.dump(node))
    if isinstance(node, ast.UnaryOp) and isinstance(node.op, ast.USub):
        return {k: -v for k, v in p_eval(node.operand, env).items()}
    if isinstance(node, ast.Constant):
        return {(): literal(node)}
    if isinstance(node, ast.Name):
        return env[node.id] if node.id in env else {(node.id,): Fraction(1)}
    if isinstance(node, ast.Subscript):
        return {(f"{node.value.id}[{node.slice.value}]",): Fraction(1)}
    if isinstance(node, ast.Call) and node.func.id == "pow":
        base = p_eval(node.args[0], env)
        e = int(ast.get_source_segment(literal.src, node.args[1]))
        r = {(): Fraction(1)}
        for _ in range(e):
            r = p_mul(r, base)
        return r
    raise ValueError(ast.dump(node))


def parse_poly(expr: str, env=None):
    literal.src = expr
    return p_eval(ast.parse(expr, mode="eval").body, env or {})


# ----------------------------------------------------------------------------
# angular basis functions
# ----------------------------------------------------------------------------
def lm_of(i):
    l = (math.isqrt(8 * i + 1) - 1) // 2
    return l, i - l * (l + 1) // 2


def harmonic(mono, which):
    """(l, m, cs) of the factor of molecule `which` (1 or 2) of a monomial."""
    l = m = 0
    cs = 0
    mt = 0
    for s in mono:
        if s.startswith(f"LegP{which}["):
            l, m = lm_of(int(s[6:-1]))
        elif s == f"cosT{which}":
            l, m = 1, 0
        elif s.startswith(f"cosP{which}_"):
            mt, cs = int(s.split("_")[1]), 0
        elif s.startswith(f"sinP{which}_"):
            mt, cs = int(s.split("_")[1]), 1
    if mt != m:
        raise ValueError(f"trig order {mt} != Legendre order {m} in {mono}")
    return l, m, cs


def code(l, m, cs):
    return 2 * (l * (l + 1) // 2 + m) + cs


def parse_basis(src):
    funcs = re.findall(r"static void (idsbf_\w+)\(Eigen::Ref<Eigen::Vector3cd> bf\) \{(.*?)\n\}", src, re.S)
    out = {}
    for name, body in funcs:
        env, comps = {}, {}
        for st in body.split(";"):
            st = st.strip()
            if not st or st.startswith("double "):
                continue
            lhs, rhs = st.split("=", 1)
            lhs = lhs.strip()
            p = parse_poly(rhs.strip(), env)
            if lhs.startswith("bf["):
                comps[int(lhs[3])] = p
            else:
                env[lhs] = p
        out[name] = comps
    return out


def dipole_order(src):
    """basis names in the order dipole_vector sums them, each with its radial function"""
    body = src[src.index("void dipole_vector(double *q, double dip[3])"):]
    body = body[:body.index("dip[0] = res(0);")]
    return re.findall(r"(idsbf_\w+)\(tmp\);\s*res \+= tmp\.real\(\) \* (radcoeff_\w+)\(R\);", body)


# ----------------------------------------------------------------------------
# radial functions
# ----------------------------------------------------------------------------
def match_paren(s, i):
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    return -1


def split_ternary(expr):
    """'R < k ? A : B' (outermost, parenthesised pieces) -> (k, A, B) or None"""
    expr = expr.strip()
    while expr.startswith("(") and match_paren(expr, 0) == len(expr) - 1:
        expr = expr[1:-1].strip()
    m = re.match(r"R < ([0-9.e+-]+) \?", expr)
    if not m:
        return None
    rest = expr[m.end():]
    depth = 0
    for i, ch in enumerate(rest):
        if ch in "(?":
            depth += 1  # a nested ternary's '?' pairs with its ':'
        elif ch == ")":
            depth -= 1
        elif ch == ":" and depth == 0:
            return m.group(1), rest[:i].strip(), rest[i + 1:].strip()
        elif ch == ":":
            depth -= 1
    raise ValueError("unbalanced ternary")


def poly_in_R(expr):
    """exact coefficients [c0, c1, ...] of a polynomial in R"""
    p = parse_poly(expr)
    deg = max((len(k) for k in p), default=0)
    c = [Fraction(0)] * (deg + 1)
    for k, v in p.items():
        if any(s != "R" for s in k):
            raise ValueError(f"unexpected symbol in radial piece: {k}")
        c[len(k)] += v
    return c


def shift(c, x0):
    """coefficients of p(x + x0) in powers of x, exactly"""
    n = len(c)
    out = [Fraction(0)] * n
    for j in range(n):
        for i in range(j, n):
            out[j] += c[i] * math.comb(i, j) * x0 ** (i - j)
    return out


def parse_radial(body):
    """-> (upper bounds, centres, [4 coefficients per piece]) of one radcoeff body"""
    k30, inner, tail = split_ternary(body)
    assert Fraction(k30) == 30
    bounds, pieces = [], []
    e = inner
    while True:
        t = split_ternary(e)
        if t is None:
            pieces.append(e)
            break
        k, a, e = t
        bounds.append(Fraction(k))
        pieces.append(a)
    centres = [Fraction("4.75")] + bounds
    bounds.append(Fraction(30))
    coefs = []
    for centre, piece in zip(centres, pieces):
        c = (poly_in_R(piece) + [Fraction(0)] * 4)[:4]
        coefs.append(shift(c, centre))
    # tail: scale * (quadratic) * pow(R, -6), or zero
    tail_s = tail.strip()
    if "pow(R, -6)" in tail_s:
        core = tail_s[: tail_s.rindex("* pow(R, -6)")].rstrip()
        core = core + ")" * (core.count("(") - core.count(")"))
        c = poly_in_R(core)
    else:
        c = poly_in_R(tail_s.rstrip(")").strip() or "0")
        assert all(v == 0 for v in c), "non-zero tail without an R^-6 factor"
    c = (c + [Fraction(0)] * 4)[:4]
    assert c[3] == 0
    coefs.append(shift(c, Fraction(30)))
    return bounds, centres + [Fraction(30)], coefs


def c_expr_value(expr, R):
    """direct float evaluation of a C radial expression (checking only)"""
    t = split_ternary(expr)
    if t is not None:
        k, a, b = t
        return c_expr_value(a, R) if R < float(k) else c_expr_value(b, R)
    return eval(expr, {"pow": pow, "R": R})


def legendre(lmax, x):
    """GSL_SF_LEGENDRE_NONE with the Condon-Shortley phase, index l(l+1)/2 + m"""
    s = math.sqrt((1 - x) * (1 + x))
    P = [0.0] * ((lmax + 1) * (lmax + 2) // 2)
    pmm = 1.0
    for m in range(lmax + 1):
        if m > 0:
            pmm *= -(2 * m - 1) * s
        P[m * (m + 1) // 2 + m] = pmm
        if m + 1 <= lmax:
            p1 = x * (2 * m + 1) * pmm
            P[(m + 1) * (m + 2) // 2 + m] = p1
            p0 = pmm
            for l in range(m + 2, lmax + 1):
                pl = ((2 * l - 1) * x * p1 - (l + m - 1) * p0) / (l - m)
                P[l * (l + 1) // 2 + m] = pl
                p0, p1 = p1, pl
    return P


def main():
    ref, out = sys.argv[1], sys.argv[2]
    src = open(f"{ref}/{SRC}").read()
    basis = parse_basis(src)
    order = dipole_order(src)
    assert len(order) == 320 and len(basis) == 320
    rad_src = dict(re.findall(r"static double (radcoeff_\w+)\(double R\) \{\s*return (.*?);\s*\}", src, re.S))
    assert len(rad_src) == 320

    rad, grid = [], None
    for _, rname in order:
        bounds, centres, coefs = parse_radial(rad_src[rname])
        if grid is None:
            grid = (bounds, centres)
        assert (bounds, centres) == grid, "radial functions on different grids"
        rad.append(coefs)
    bounds, centres = grid
    nseg = len(centres)

    terms = []  # (coef, b, comp, y1, y2)
    for b, (bname, _) in enumerate(order):
        for comp in range(3):
            for mono, v in sorted(basis[bname].get(comp, {}).items()):
                l1, m1, c1 = harmonic(mono, 1)
                l2, m2, c2 = harmonic(mono, 2)
                if float(v) != 0.0:
                    terms.append((v, b, comp, code(l1, m1, c1), code(l2, m2, c2)))

    # ---- checks against the source's own expressions ----
    rng = random.Random(5)

    def seg_of(R):
        for i, hi in enumerate(bounds):
            if R < hi:
                return i
        return nseg - 1

    for _ in range(400):
        R = rng.uniform(3.5, 45.0)
        b = rng.randrange(320)
        s = seg_of(R)
        x = R - float(centres[s])
        c = [float(v) for v in rad[b][s]]
        val = c[0] + x * (c[1] + x * (c[2] + x * c[3]))
        if s == nseg - 1:
            val *= R ** -6
        ref_val = c_expr_value(rad_src[order[b][1]], R)
        assert abs(val - ref_val) <= 1e-11 * max(1.0, abs(ref_val)), (b, R, val, ref_val)

    for _ in range(20):
        th1, th2 = rng.uniform(0.1, 3.0), rng.uniform(0.1, 3.0)
        ph1, ph2 = rng.uniform(-3, 3), rng.uniform(-3, 3)
        env = {"cosT1": math.cos(th1), "cosT2": math.cos(th2)}
        L1, L2 = legendre(16, math.cos(th1)), legendre(12, math.cos(th2))
        for k in range(1, 14):
            env[f"cosP1_{k}"], env[f"sinP1_{k}"] = math.cos(k * ph1), math.sin(k * ph1)
            env[f"cosP2_{k}"], env[f"sinP2_{k}"] = math.cos(k * ph2), math.sin(k * ph2)
        for i, v in enumerate(L1):
            env[f"LegP1[{i}]"] = v
        for i, v in enumerate(L2):
            env[f"LegP2[{i}]"] = v
        b = rng.randrange(320)
        bname = order[b][0]
        body = re.search(r"static void " + bname + r"\(Eigen::Ref<Eigen::Vector3cd> bf\) \{(.*?)\n\}", src, re.S).group(1)
        loc, direct = {}, [0.0, 0.0, 0.0]
        for st in body.split(";"):
            st = st.strip()
            if not st or st.startswith("double "):
                continue
            lhs, rhs = st.split("=", 1)
            e = re.sub(r"(LegP[12]\[\d+\]|cosP[12]_\d+|sinP[12]_\d+|cosT[12])", lambda mm: repr(env[mm.group(1)]), rhs)
            v = eval(e, {}, loc)
            lhs = lhs.strip()
            if lhs.startswith("bf["):
                direct[int(lhs[3])] = v
            else:
                loc[lhs] = v

        def hv(cd, which):
            i, cs = cd // 2, cd % 2
            _, m = lm_of(i)
            P = (L1 if which == 1 else L2)[i]
            ph = ph1 if which == 1 else ph2
            if m == 0:
                return P
            return P * (math.cos(m * ph) if cs == 0 else math.sin(m * ph))

        exp = [0.0, 0.0, 0.0]
        for (v, bb, comp, y1, y2) in terms:
            if bb == b:
                exp[comp] += float(v) * hv(y1, 1) * hv(y2, 2)
        scale = max(1e-30, max(abs(t) for t in direct))
        assert max(abs(exp[c] - direct[c]) for c in range(3)) <= 1e-12 * scale, (bname, exp, direct)

    l1max = max(lm_of(t[3] // 2)[0] for t in terms)
    l2max = max(lm_of(t[4] // 2)[0] for t in terms)

    def fx(v):
        return repr(float(v))

    with open(out, "w") as f:
        f.write("// Generated by gen_ch4co2_tables.py from the reference tree's\n")
        f.write("// PES-IDS/ai_ids_ch4_co2.cpp (dipole_vector, lines 672-1067); do not edit.\n")
        f.write("// Radial functions: piece s covers R < hh_ch4co2_seg_hi[s] above the previous\n")
        f.write("// bound (piece 0 extends down, the last piece, R >= 30, up); value =\n")
        f.write("// c0 + x (c1 + x (c2 + x c3)), x = R - hh_ch4co2_centre[s], times R^-6 on the last\n")
        f.write("// piece.  Terms: mu_c += coef * rad_b(R) * Y1 * Y2 with\n")
        f.write("// Y = P_l^m(cos theta) * (m == 0 ? 1 : cs ? sin(m phi) : cos(m phi)),\n")
        f.write("// harmonic code 2 * (l(l+1)/2 + m) + cs.\n")
        f.write("#pragma once\n\n")
        f.write(f"#define HH_CH4CO2_NB 320\n#define HH_CH4CO2_NSEG {nseg}\n#define HH_CH4CO2_NTERM {len(terms)}\n")
        f.write(f"#define HH_CH4CO2_L1MAX {l1max}\n#define HH_CH4CO2_L2MAX {l2max}\n\n")
        f.write(f"static const double hh_ch4co2_seg_hi[{nseg - 1}] = {{{', '.join(fx(v) for v in bounds)}}};\n")
        f.write(f"static const double hh_ch4co2_centre[{nseg}] = {{{', '.join(fx(v) for v in centres)}}};\n\n")
        f.write(f"static const double hh_ch4co2_rad[320][{nseg}][4] = {{\n")
        for b in range(320):
            f.write("  {" + ", ".join("{" + ", ".join(fx(v) for v in rad[b][s]) + "}" for s in range(nseg)) + "},\n")
        f.write("};\n\n")
        f.write(f"static const double hh_ch4co2_tcoef[{len(terms)}] = {{\n")
        for i in range(0, len(terms), 4):
            f.write("  " + ", ".join(fx(t[0]) for t in terms[i:i + 4]) + ",\n")
        f.write("};\n\n")
        f.write(f"// b, component, Y1 code, Y2 code\nstatic const short hh_ch4co2_tidx[{len(terms)}][4] = {{\n")
        for i in range(0, len(terms), 8):
            f.write("  " + ", ".join(f"{{{t[1]}, {t[2]}, {t[3]}, {t[4]}}}" for t in terms[i:i + 8]) + ",\n")
        f.write("};\n")
    print(f"wrote {out}: {len(terms)} terms, {nseg} radial pieces, l1 <= {l1max}, l2 <= {l2max}")


if __name__ == "__main__":
    main()
