"""Write the DOP853 Butcher tableau as a C header.

DOP853 is the explicit embedded Runge-Kutta pair of order 8(5,3) with a
7th-order continuous extension published by Hairer, Norsett and Wanner
("Solving Ordinary Differential Equations I", 2nd ed., Sec. II.10).  Its
coefficients are taken from SciPy's transcription of that publication
(``scipy.integrate._ivp.dop853_coefficients``), printed with full double
precision so that the CUDA kernels and the CPU oracle share one tableau.

Usage: python gen_dop853_tableau.py <output header>
"""
import sys

from scipy.integrate._ivp import dop853_coefficients as dc


def arr(name, a):
    return f"HH_TAB_QUAL double {name}[{len(a)}] = {{" + ", ".join(repr(float(x)) for x in a) + "};\n"


def main():
    out = sys.argv[1]
    A = dc.A
    with open(out, "w") as fh:
        fh.write("/* Generated by gen_dop853_tableau.py (DOP853 of Hairer, Norsett and Wanner).  Do not edit. */\n")
        fh.write("#pragma once\n\n")
        fh.write("#if defined(__CUDACC__)\n#define HH_TAB_QUAL static constexpr __device__\n"
                 "#elif defined(__cplusplus)\n#define HH_TAB_QUAL static constexpr\n"
                 "#else\n#define HH_TAB_QUAL static const\n#endif\n\n")
        fh.write(f"#define HH_DOP853_NSTAGES {dc.N_STAGES}\n#define HH_DOP853_NSTAGES_EXT {dc.N_STAGES_EXTENDED}\n\n")
        fh.write(arr("hh_dop853_c", dc.C))
        fh.write(f"HH_TAB_QUAL double hh_dop853_a[{A.shape[0]}][{A.shape[1]}] = {{\n")
        for row in A:
            fh.write("  {" + ", ".join(repr(float(x)) for x in row) + "},\n")
        fh.write("};\n")
        fh.write(arr("hh_dop853_e3", dc.E3))
        fh.write(arr("hh_dop853_e5", dc.E5))
        fh.write(f"HH_TAB_QUAL double hh_dop853_d[{dc.D.shape[0]}][{dc.D.shape[1]}] = {{\n")
        for row in dc.D:
            fh.write("  {" + ", ".join(repr(float(x)) for x in row) + "},\n")
        fh.write("};\n")


if __name__ == "__main__":
    main()
