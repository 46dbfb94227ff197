#!/usr/bin/env python3
"""Generate hh_mt_jump.h: jump-ahead tables for the MT19937 stream.

The MT19937 recurrence x[n+624] = x[n+397] ^ twist(upper(x[n]) | lower(x[n+1])) is
linear over GF(2) on the 19,937 bits of a 624-word window W(m) = x[m .. m+623]
(the 31 low bits of x[m] are not part of the state).  With phi the characteristic
polynomial of the one-word shift A: W(m) -> W(m+1) and p(x) = x^J mod phi(x),
A^J = p(A), so

    W(m + J) = XOR over the set bits i of p of W(m + i),

i.e. word j of the window J words ahead is the XOR of x[m + i + j] over those i
(Haramoto et al., "Efficient jump ahead for F2-linear random number generators",
INFORMS J. Computing 20 (2008)).  It needs the 19,937 + 623 words that follow m.

phi is found by the Berlekamp-Massey algorithm on one bit of the untempered
stream (phi is primitive, so the minimal polynomial of any non-zero bit sequence
is phi itself).  The script writes the positions of the set bits of x^J mod phi
for J = HH_MT_SEG_WORDS and J = HH_MT_COARSE * HH_MT_SEG_WORDS, and checks both
jumps against direct simulation of the stream before it writes the header.  It also
writes x^(k J) mod phi for J = HH_MT_SEG_WORDS and k = 1 .. HH_MT_COARSE - 1 (the
"fine" table), so that every segment of a coarse interval is one jump from the
interval's start (the products are checked for k = 2 and k = 3 against the stream).

usage: gen_mt_jump.py <output header>
"""
from __future__ import annotations

import sys

import numpy as np

N, M = 624, 397
MATRIX_A = np.uint32(0x9908B0DF)
UPPER, LOWER = np.uint32(0x80000000), np.uint32(0x7FFFFFFF)
DEG = 19937
SEG_BLOCKS = 2048               # 624-word blocks per generated segment
SEG_WORDS = SEG_BLOCKS * N
COARSE = 32                     # segments per coarse jump


def seed_state(seed: int) -> np.ndarray:
    """Knuth 69069 seeding as mtwist's mts_seed32 does (state before its first refresh)."""
    s = np.empty(N, dtype=np.uint64)
    s[0] = seed
    for i in range(1, N):
        s[i] = (69069 * int(s[i - 1])) & 0xFFFFFFFF
    return s.astype(np.uint32)


def twist(a, b, c):
    y = (a & UPPER) | (b & LOWER)
    return c ^ (y >> np.uint32(1)) ^ np.where((y & np.uint32(1)) != 0, MATRIX_A, np.uint32(0)).astype(np.uint32)


def refresh(block: np.ndarray) -> np.ndarray:
    """next 624 untempered words after the window `block` (three dependency phases)"""
    new = np.empty(N, dtype=np.uint32)
    k = N - M  # 227
    new[:k] = twist(block[:k], block[1:k + 1], block[M:])
    new[k:2 * k] = twist(block[k:2 * k], block[k + 1:2 * k + 1], new[:k])
    i = np.arange(2 * k, N)
    nxt = np.where(i + 1 < N, block[np.minimum(i + 1, N - 1)], new[0])
    new[2 * k:] = twist(block[2 * k:], nxt, new[i - k])
    return new


def stream(state: np.ndarray, nblocks: int) -> np.ndarray:
    out = np.empty(nblocks * N, dtype=np.uint32)
    cur = state
    for b in range(nblocks):
        cur = refresh(cur)
        out[b * N:(b + 1) * N] = cur
    return out


def berlekamp_massey(bits: list[int]) -> int:
    """connection polynomial C(x) (bit i = c_i, c_0 = 1) of a GF(2) sequence"""
    n = len(bits)
    R = 0
    for k, b in enumerate(bits):
        if b:
            R |= 1 << (n - 1 - k)
    C, B, L, m = 1, 1, 0, 1
    for i in range(n):
        d = bin((R >> (n - 1 - i)) & C).count("1") & 1
        if d == 0:
            m += 1
        elif 2 * L <= i:
            T = C
            C ^= B << m
            L = i + 1 - L
            B = T
            m = 1
        else:
            C ^= B << m
            m += 1
    return C, L


# byte v -> the 16-bit value with bit 2k = bit k of v (squaring in GF(2)[x])
_SPREAD = [int("".join("0" + c for c in format(v, "08b")), 2) for v in range(256)]


def gf2_square(a: int) -> int:
    out = 0
    shift = 0
    while a:
        out |= _SPREAD[a & 0xFF] << shift
        a >>= 8
        shift += 16
    return out


def gf2_mod(a: int, phi: int, deg: int) -> int:
    while a.bit_length() - 1 >= deg:
        a ^= phi << (a.bit_length() - 1 - deg)
    return a


def x_pow_mod(J: int, phi: int, deg: int) -> int:
    r = 1
    for bit in bin(J)[2:]:
        r = gf2_mod(gf2_square(r), phi, deg)
        if bit == "1":
            r = gf2_mod(r << 1, phi, deg)
    return r


def gf2_mulmod(a: int, b: int, phi: int, deg: int) -> int:
    """a * b mod phi in GF(2)[x]"""
    r = 0
    i = 0
    while a:
        if a & 1:
            r ^= b << i
        a >>= 1
        i += 1
    return gf2_mod(r, phi, deg)


def jump(words: np.ndarray, m: int, p: int) -> np.ndarray:
    """W(m + J) from the stream words following position m"""
    acc = np.zeros(N, dtype=np.uint32)
    i = 0
    while p:
        if p & 1:
            acc ^= words[m + i:m + i + N]
        p >>= 1
        i += 1
    return acc


def main():
    out = sys.argv[1]
    st = seed_state(5489)
    w = stream(st, 2 * DEG // N + 4)
    bits = [int(x) & 1 for x in w[:2 * DEG]]
    C, L = berlekamp_massey(bits)
    assert L == DEG, L
    # characteristic polynomial: the reciprocal of the connection polynomial
    phi = int(format(C, f"0{DEG + 1}b")[::-1], 2)
    assert phi >> DEG == 1
    tables = {}
    for name, J in (("seg", SEG_WORDS), ("coarse", COARSE * SEG_WORDS)):
        p = x_pow_mod(J, phi, DEG)
        tables[name] = [i for i in range(DEG) if (p >> i) & 1]
        # check: W(m + J) for m = 0 (window of the first 624 stream words) against the stream
        need = J // N + 2
        full = stream(st, need + 1)
        got = jump(full, 0, p)
        want = full[J:J + N]
        mask = np.full(N, 0xFFFFFFFF, dtype=np.uint32)
        mask[0] = 0x80000000     # the low 31 bits of the window's first word are not state
        assert np.array_equal(got & mask, want & mask), name
        print(f"{name}: J = {J} words, {len(tables[name])} set bits, checked against the stream")
    # the fine table: x^(k SEG) mod phi, k = 1 .. COARSE - 1
    p1 = x_pow_mod(SEG_WORDS, phi, DEG)
    fine = [p1]
    for k in range(2, COARSE):
        fine.append(gf2_mulmod(fine[-1], p1, phi, DEG))
    for k in (2, 3):
        J = k * SEG_WORDS
        full = stream(st, J // N + 3)
        got = jump(full, 0, fine[k - 1])
        mask = np.full(N, 0xFFFFFFFF, dtype=np.uint32)
        mask[0] = 0x80000000
        assert np.array_equal(got & mask, full[J:J + N] & mask), k
        print(f"fine k = {k}: checked against the stream")
    fine_bits = [[i for i in range(DEG) if (p >> i) & 1] for p in fine]
    assert fine_bits[0] == tables["seg"]
    fine_max = max(len(t) for t in fine_bits)
    with open(out, "w") as f:
        f.write("// Generated by gen_mt_jump.py; do not edit.  Jump-ahead tables of the MT19937\n")
        f.write("// stream: the set bits i of x^J mod phi(x), so that the 624-word window J words\n")
        f.write("// ahead of position m is the XOR of the windows at m + i (see the generator).\n")
        f.write("#pragma once\n\n")
        f.write(f"#define HH_MT_SEG_BLOCKS {SEG_BLOCKS}\n#define HH_MT_COARSE {COARSE}\n")
        for name in ("seg", "coarse"):
            t = tables[name]
            f.write(f"#define HH_MT_JUMP_{name.upper()}_N {len(t)}\n")
            f.write(f"static const unsigned short hh_mt_jump_{name}[{len(t)}] = {{\n")
            for k in range(0, len(t), 16):
                f.write("  " + ", ".join(str(v) for v in t[k:k + 16]) + ",\n")
            f.write("};\n")
        f.write(f"#define HH_MT_JUMP_FINE_MAX {fine_max}\n")
        f.write(f"static const unsigned short hh_mt_jump_fine_n[{COARSE - 1}] = {{"
                + ", ".join(str(len(t)) for t in fine_bits) + "};\n")
        f.write(f"static const unsigned short hh_mt_jump_fine[{COARSE - 1}][{fine_max}] = {{\n")
        for t in fine_bits:
            f.write("  {\n")
            for k in range(0, len(t), 16):
                f.write("    " + ", ".join(str(v) for v in t[k:k + 16]) + ",\n")
            f.write("  },\n")
        f.write("};\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
