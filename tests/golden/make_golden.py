"""Build the golden fixtures used by the test suite from the reference checkout.

Run once where the reference checkout is present:
    python tests/golden/make_golden.py <reference checkout>
(or with the checkout in the environment variable HH_REFERENCE_DIR).
Writes tests/golden/cf_sf_he_ar_1000.npz from the reference's own golden pair
(tests/CF-F-He-Ar-1000.0.txt -> tests/SF-F-He-Ar-1000.0.txt, produced by the
reference's CF_TO_SF, tests/convert-cf-to-sf.conf:6-9): the CF time grid and
values, the SF frequency grid and values, and the header fields.
"""
import os
import sys

import numpy as np


def read_table(path):
    header = {}
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("# AVERAGE OVER"):
                header["NTRAJ"] = float(line.split()[3])
                continue
            if line.startswith("#"):
                if ":" in line:
                    k, v = line[1:].split(":", 1)
                    header[k.strip()] = v.strip()
                continue
            a, b = line.split()
            rows.append((float(a), float(b)))
    return header, np.array(rows)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HH_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set HH_REFERENCE_DIR)")
    hcf, cf = read_table(os.path.join(ref, "tests", "CF-F-He-Ar-1000.0.txt"))
    hsf, sf = read_table(os.path.join(ref, "tests", "SF-F-He-Ar-1000.0.txt"))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cf_sf_he_ar_1000.npz")
    ntraj = hcf["NTRAJ"]
    dt = cf[1, 0] - cf[0, 0]
    assert np.array_equal(cf[:, 0], dt * np.arange(cf.shape[0]))
    np.savez_compressed(
        out,
        dt=dt, cf=cf[:, 1], sf=sf[:, 1],
        sf_nu_every64=sf[::64, 0],
        temperature=float(hcf["TEMPERATURE"]),
        ntraj=ntraj,
    )
    print("wrote", out, os.path.getsize(out), "bytes")


def make_ref_surfaces():
    """tests/golden/ref_surfaces.npz from the reference sources compiled in oracle/_ref
    (thirdparty/mtwist.c, PES-IDS/HeAr.h, PES-IDS/ai_pes_co2ar.c, PES-IDS/ai_ids_co2ar.cpp)."""
    import ctypes as C
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, root)
    from oracle import oracle as O
    O.build()
    mt = O.ref("mtwist")
    words = {}
    for seed in (42, 7, 1):
        mt.mt_seed32(seed)
        words[seed] = np.array([mt.mt_lrand() for _ in range(4000)], dtype=np.uint32)
    h = O.ref("hear")
    R = np.linspace(3.0, 45.0, 421)
    he = np.array([[h.V_HeAr(r), h.dV_HeAr(r), h.dip_HeAr(r)] for r in R])
    pes, ids = O.ref("co2ar_pes"), O.ref("co2ar_ids")
    rng = np.random.default_rng(2024)
    Rc = np.concatenate([rng.uniform(3.5, 45.0, 3000), np.array([4.5, 4.75, 10.0, 20.0, 25.0, 30.0, 6.4966051519])])
    Th = np.concatenate([np.arccos(rng.uniform(-1.0, 1.0, 3000)), np.full(7, np.pi / 2)])
    co = []
    for r, t in zip(Rc, Th):
        a, b = C.c_double(), C.c_double()
        pes.dpes_co2ar(r, t, a, b)
        d = np.zeros(3)
        ids.ref_co2ar_dip_mol(r, t, d)
        co.append([pes.pes_co2ar(r, t), a.value, b.value, d[0], d[2]])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_surfaces.npz")
    np.savez_compressed(out, mt42=words[42], mt7=words[7], mt1=words[1], hear_R=R, hear=he,
                        co2ar_R=Rc, co2ar_theta=Th, co2ar=np.array(co))
    print("wrote", out, os.path.getsize(out), "bytes")


def make_ch4co2_dipole():
    """tests/golden/ref_ch4co2_dipole.npz: the reference's CH4-CO2 dipole chain compiled in
    oracle/_ref (PES-IDS/ai_ids_ch4_co2.cpp, PES-IDS/ai_ids_ch4_co2_lib.cpp,
    src/angles_handler.cpp) at seeded lab-frame points (PHI THETA R PHI1 THETA1 PSI1 PHI2 THETA2):
    the molecular-frame coordinates, the body-frame dipole and the lab-frame dipole."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sys.path.insert(0, root)
    from oracle import oracle as O
    O.build()
    L = O.ref("ch4co2_ids")
    rng = np.random.default_rng(4096)
    n = 600
    R = np.concatenate([rng.uniform(4.0, 45.0, n - 8), [4.75, 5.0, 9.5, 10.0, 25.0, 29.999, 30.0, 40.0]])
    q = np.column_stack([rng.uniform(0, 2 * np.pi, n), np.arccos(rng.uniform(-1, 1, n)), R,
                         rng.uniform(0, 2 * np.pi, n), np.arccos(rng.uniform(-1, 1, n)),
                         rng.uniform(0, 2 * np.pi, n), rng.uniform(0, 2 * np.pi, n),
                         np.arccos(rng.uniform(-1, 1, n))])
    kal = np.zeros((n, 5))
    dk = np.zeros((n, 3))
    dl = np.zeros((n, 3))
    for i in range(n):
        L.ref_ch4co2_lab_to_kal(np.ascontiguousarray(q[i]), kal[i])
        L.ref_ch4co2_dipole_vector(np.ascontiguousarray(kal[i]), dk[i])
        L.ref_ch4co2_dipole_lab(np.ascontiguousarray(q[i]), dl[i])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_ch4co2_dipole.npz")
    np.savez_compressed(out, q=q, kal=kal, dip_kal=dk, dip_lab=dl)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
    make_ref_surfaces()
    make_ch4co2_dipole()
