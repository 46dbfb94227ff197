#!/usr/bin/env python3
"""Generate hh_n2ar_tables.h: the N2-Ar PIP-NN surfaces as data.

Reads, from a HAWAIIHYBRID source tree:
  PES-IDS/c_basis_2_1_4_purify.cc          17 permutationally invariant polynomials
                                           (PIPs) of the 3 N2-Ar distance variables
  PES-IDS/c_basis_1_1_2_1_3_purify.cc,     119 + 119 + 70 PIPs of the 10 distance
  PES-IDS/c_basis_2_1_1_1_3_purify.cc,     variables of the 5-site dipole model, in the
  PES-IDS/c_basis_2_2_1_3_purify.cc        order PES-IDS/ai_ids_n2_ar_pip_nn.cpp:41-48 uses
  PES-IDS/npz/n2-ar-nonrigid-17-32-1-f12.npz      PES MLP (mlp.hpp)
  PES-IDS/npz/n2-ar-dipoleq-effquad-{short,long}.npz  dipole charge models (QModel.hpp)

and writes each PIP basis as a table of monomials (variable indices, -1 padded)
with the PIP each monomial adds into, plus the network weights in the (in, out)
orientation the reference multiplies with (row vector times matrix).  Every
polynomial of these bases is a sum of monomials with coefficient 1.

usage: gen_n2ar_tables.py <reference-root> <output header>
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

PES_BASIS = "c_basis_2_1_4_purify.cc"
DIP_BASES = ("c_basis_1_1_2_1_3_purify.cc", "c_basis_2_1_1_1_3_purify.cc", "c_basis_2_2_1_3_purify.cc")
PES_NPZ = "n2-ar-nonrigid-17-32-1-f12.npz"
DIP_NPZ = ("n2-ar-dipoleq-effquad-short.npz", "n2-ar-dipoleq-effquad-long.npz")


def parse_basis(path: str):
    """-> (npoly, [(poly, (var, var, ...)), ...]) from `p(i) = y[a]*y[b] + ...;` lines."""
    src = open(path).read()
    src = re.sub(r"//[^\n]*", "", src)
    body = src[src.index("{") + 1:]
    npoly = 0
    monos = []
    for idx, rhs in re.findall(r"p\((\d+)\)\s*=\s*([^;]+);", body):
        i = int(idx)
        npoly = max(npoly, i + 1)
        rhs = " ".join(rhs.split())
        if re.fullmatch(r"0(\.0*)?", rhs):
            continue  # identically zero polynomial
        for term in rhs.split("+"):
            vars_ = []
            for fac in term.split("*"):
                fac = fac.strip()
                m = re.fullmatch(r"y\[(\d+)\]", fac)
                if not m:
                    raise ValueError(f"{path}: unexpected factor {fac!r} in p({i})")
                vars_.append(int(m.group(1)))
            monos.append((i, tuple(sorted(vars_))))
    return npoly, monos


def fmt(v) -> str:
    return repr(float(v))


def emit_array(fh, ctype, name, arr):
    arr = np.asarray(arr)
    dims = "".join(f"[{d}]" for d in arr.shape)
    fh.write(f"HH_TAB_QUAL {ctype} {name}{dims} = ")
    if arr.ndim == 1:
        fh.write("{" + ", ".join(fmt(x) if ctype == "double" else str(int(x)) for x in arr) + "};\n")
    else:
        rows = []
        for row in arr:
            rows.append("  {" + ", ".join(fmt(x) if ctype == "double" else str(int(x)) for x in row) + "}")
        fh.write("{\n" + ",\n".join(rows) + "\n};\n")


def mono_table(monos, width):
    vars_ = np.full((len(monos), width), -1, dtype=np.int64)
    polys = np.zeros(len(monos), dtype=np.int64)
    for k, (p, v) in enumerate(monos):
        vars_[k, :len(v)] = v
        polys[k] = p
    return vars_, polys


def main():
    ref, out = sys.argv[1], sys.argv[2]
    pes_dir = os.path.join(ref, "PES-IDS")
    npz_dir = os.path.join(pes_dir, "npz")
    with open(out, "w") as fh:
        fh.write("/* Generated by gen_n2ar_tables.py from the HAWAIIHYBRID N2-Ar PIP-NN surfaces\n"
                 " * (PES-IDS/c_basis_*_purify.cc, PES-IDS/npz/n2-ar-*.npz).  Do not edit. */\n")
        fh.write("#pragma once\n\n#if defined(__CUDACC__)\n#define HH_TAB_QUAL static constexpr __device__\n"
                 "#elif defined(__cplusplus)\n#define HH_TAB_QUAL static constexpr\n#else\n"
                 "#define HH_TAB_QUAL static const\n#endif\n\n")
        # ---- PES basis ----
        npoly, monos = parse_basis(os.path.join(pes_dir, PES_BASIS))
        v, p = mono_table(monos, 4)
        fh.write(f"/* PES: {npoly} PIPs of y[0..2]; monomial k adds prod_j y[var[k][j]] into PIP poly[k] */\n")
        fh.write(f"#define HH_N2AR_PES_NPIP {npoly}\n#define HH_N2AR_PES_NMONO {len(monos)}\n")
        emit_array(fh, "signed char", "hh_n2ar_pes_var", v)
        emit_array(fh, "unsigned char", "hh_n2ar_pes_poly", p)
        # ---- dipole bases ----
        allm = []
        off = 0
        sizes = []
        for b in DIP_BASES:
            n, m = parse_basis(os.path.join(pes_dir, b))
            allm += [(off + i, vv) for i, vv in m]
            sizes.append(n)
            off += n
        v, p = mono_table(allm, 3)
        fh.write(f"\n/* dipole: {off} PIPs of y[0..9] ({' + '.join(map(str, sizes))}, one block per sub-network) */\n")
        fh.write(f"#define HH_N2AR_DIP_NPIP {off}\n#define HH_N2AR_DIP_NMONO {len(allm)}\n")
        fh.write("".join(f"#define HH_N2AR_DIP_NPIP{i} {n}\n" for i, n in enumerate(sizes)))
        emit_array(fh, "signed char", "hh_n2ar_dip_var", v)
        emit_array(fh, "short", "hh_n2ar_dip_poly", p)
        # ---- PES network ----
        z = np.load(os.path.join(npz_dir, PES_NPZ))
        arch = [int(a) for a in z["architecture"]]
        if arch != [npoly, 32, 1]:
            raise ValueError(f"unexpected PES architecture {arch}")
        fh.write(f"\n/* PES network {arch[0]}-{arch[1]}-{arch[2]}: E = yscale * (SiLU(ptr W0 + b0) W1 + b1) + ymean,\n"
                 " * ptr = (p - xmean) / xscale; E in cm^-1 */\n")
        fh.write(f"#define HH_N2AR_PES_HIDDEN {arch[1]}\n")
        emit_array(fh, "double", "hh_n2ar_pes_xmean", z["xscaler.mean"])
        emit_array(fh, "double", "hh_n2ar_pes_xscale", z["xscaler.scale"])
        emit_array(fh, "double", "hh_n2ar_pes_y", [z["yscaler.mean"][0], z["yscaler.scale"][0]])
        emit_array(fh, "double", "hh_n2ar_pes_w0", z["0.weight"])
        emit_array(fh, "double", "hh_n2ar_pes_b0", z["0.bias"])
        emit_array(fh, "double", "hh_n2ar_pes_w1", z["2.weight"][:, 0])
        emit_array(fh, "double", "hh_n2ar_pes_b1", z["2.bias"])
        # ---- dipole charge models, flattened: sub-network s of model m has its
        # first-layer rows at w0[m][W0OFF[s] ...] ([nin][nhid] row-major), its
        # hidden units at b0[m][B0OFF[s] ...], its output layer at w1[m][W1OFF[s] ...]
        # ([nhid][nout] row-major) and its charges at b1/qinf[m][QOFF[s] ...] ----
        archs = []
        zs = [np.load(os.path.join(npz_dir, f)) for f in DIP_NPZ]
        for s_ in range(3):
            a = [int(x) for x in zs[0][f"architecture.{s_}"]]
            for z in zs:
                if [int(x) for x in z[f"architecture.{s_}"]] != a:
                    raise ValueError("the two dipole models differ in architecture")
            if a[0] != sizes[s_]:
                raise ValueError(f"sub-network {s_} reads {a[0]} PIPs, basis has {sizes[s_]}")
            archs.append(a)
        w0off, b0off, w1off, qoff = [0], [0], [0], [0]
        for a in archs:
            w0off.append(w0off[-1] + a[0] * a[1])
            b0off.append(b0off[-1] + a[1])
            w1off.append(w1off[-1] + a[1] * a[2])
            qoff.append(qoff[-1] + a[2])
        fh.write("\n/* dipole charge models [0] = short range (a0 = 2), [1] = long range (a0 = 6)\n"
                 " * (PES-IDS/npz/n2-ar-dipoleq-effquad-{short,long}.npz); sub-network s maps PIPs\n"
                 " * [PIPOFF[s], PIPOFF[s+1]) through SiLU(ptr W0 + b0) W1 + b1 to charges\n"
                 " * [QOFF[s], QOFF[s+1]) of the sites N1, N2, N1', N2', Ar */\n")
        fh.write(f"#define HH_N2AR_DIP_NW0 {w0off[-1]}\n#define HH_N2AR_DIP_NB0 {b0off[-1]}\n"
                 f"#define HH_N2AR_DIP_NW1 {w1off[-1]}\n#define HH_N2AR_DIP_NQ {qoff[-1]}\n")
        pipoff = [0, sizes[0], sizes[0] + sizes[1], off]
        emit_array(fh, "int", "hh_n2ar_dip_arch", np.array(archs))
        emit_array(fh, "int", "hh_n2ar_dip_pipoff", pipoff)
        emit_array(fh, "int", "hh_n2ar_dip_w0off", w0off)
        emit_array(fh, "int", "hh_n2ar_dip_b0off", b0off)
        emit_array(fh, "int", "hh_n2ar_dip_w1off", w1off)
        emit_array(fh, "int", "hh_n2ar_dip_qoff", qoff)
        # CSR over the monomial table (monomials are grouped by PIP)
        polys = p
        if np.any(np.diff(polys) < 0):
            raise ValueError("dipole monomials are not grouped by PIP")
        start = np.searchsorted(polys, np.arange(off + 1), side="left")
        emit_array(fh, "short", "hh_n2ar_dip_start", start)
        W0 = np.zeros((2, w0off[-1])); B0 = np.zeros((2, b0off[-1]))
        W1 = np.zeros((2, w1off[-1])); B1 = np.zeros((2, qoff[-1]))
        XM = np.zeros((2, off)); XS = np.zeros((2, off))
        for m, z in enumerate(zs):
            XM[m] = z["xscaler.mean"]
            XS[m] = z["xscaler.scale"]
            for s_ in range(3):
                W0[m, w0off[s_]:w0off[s_ + 1]] = z[f"blocks.{s_}.0.weight"].ravel(order="C")
                B0[m, b0off[s_]:b0off[s_ + 1]] = z[f"blocks.{s_}.0.bias"]
                W1[m, w1off[s_]:w1off[s_ + 1]] = z[f"blocks.{s_}.2.weight"].ravel(order="C")
                B1[m, qoff[s_]:qoff[s_ + 1]] = z[f"blocks.{s_}.2.bias"]
        emit_array(fh, "double", "hh_n2ar_dip_xmean", XM)
        emit_array(fh, "double", "hh_n2ar_dip_xscale", XS)
        emit_array(fh, "double", "hh_n2ar_dip_w0", W0)
        emit_array(fh, "double", "hh_n2ar_dip_b0", B0)
        emit_array(fh, "double", "hh_n2ar_dip_w1", W1)
        emit_array(fh, "double", "hh_n2ar_dip_b1", B1)

if __name__ == "__main__":
    main()
