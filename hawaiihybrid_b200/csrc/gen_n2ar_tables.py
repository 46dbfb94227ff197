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
        # ---- dipole charge models ----
        for tag, f in zip(("short", "long"), DIP_NPZ):
            z = np.load(os.path.join(npz_dir, f))
            fh.write(f"\n/* dipole charge model `{tag}` ({f}): sub-network s maps its PIP block\n"
                     " * through SiLU(ptr W0 + b0) W1 + b1 to its charges */\n")
            emit_array(fh, "double", f"hh_n2ar_dip_{tag}_xmean", z["xscaler.mean"])
            emit_array(fh, "double", f"hh_n2ar_dip_{tag}_xscale", z["xscaler.scale"])
            for s in range(3):
                a = [int(x) for x in z[f"architecture.{s}"]]
                if a[0] != sizes[s]:
                    raise ValueError(f"{f}: sub-network {s} reads {a[0]} PIPs, basis has {sizes[s]}")
                fh.write(f"#define HH_N2AR_DIP_{tag.upper()}_ARCH{s} {{{a[0]}, {a[1]}, {a[2]}}}\n")
                emit_array(fh, "double", f"hh_n2ar_dip_{tag}_w0_{s}", z[f"blocks.{s}.0.weight"])
                emit_array(fh, "double", f"hh_n2ar_dip_{tag}_b0_{s}", z[f"blocks.{s}.0.bias"])
                emit_array(fh, "double", f"hh_n2ar_dip_{tag}_w1_{s}", z[f"blocks.{s}.2.weight"])
                emit_array(fh, "double", f"hh_n2ar_dip_{tag}_b1_{s}", z[f"blocks.{s}.2.bias"])


if __name__ == "__main__":
    main()
