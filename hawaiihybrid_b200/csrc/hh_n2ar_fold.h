// N2-Ar dipole charge models folded for the body frame (shared by the host
// builder hh_n2ar_host.cpp and the kernels).
//
// In the dipole model's body frame (Ar on +z at R, N1 at L/2 (sin T, 0, cos T),
// N1' at L/2 (cos T, 0, -sin T)), six of the ten site distances are fixed by the
// rigid rotor: |N1-N2| = |N1'-N2'| = L and |N-N'| = L/sqrt(2).  Only y3 (N1-Ar),
// y6 (N2-Ar), y8 (N1'-Ar) and y9 (N2'-Ar) vary, so each of the 308 PIPs is a
// polynomial of degree <= 3 in those four variables with no constant term (the
// bases are purified: every monomial contains an Ar pair).  The PIP layer, the
// input scaler and the first network layer of each charge model therefore fold
// into one matrix over the 34 monomials z_k of (y3, y6, y8, y9):
//   h(p) - h(0) = sum_k z_k w[k]          (the scaler mean cancels exactly)
// and the charges relative to infinite separation (QModel::forward_inf) are
//   q - q_inf = W1^T (SiLU(h0 + dh) - SiLU(h0))   (the output bias cancels),
// with SiLU(a + d) - SiLU(a) = s(a+d) (d - a (1 - s(a)) u), u = expm1(-d), s the
// logistic function, and s(a+d) = 1 / (1 + e^-a (1 + u)): one expm1 and one
// division per hidden unit.  The dipole needs q_N1 - q_N2 and q_N1' - q_N2', so the
// output weights are stored differenced.  Every step avoids the cancellations of
// the reference's q - q_inf, which cost FP32 about 5e-4 of the dipole.
#pragma once

constexpr int N2AR_NZ = 34;    // monomials of degree 1..3 in 4 variables
constexpr int N2AR_NH = 40;    // hidden units of the three sub-networks (16 + 16 + 8)

struct N2arDipFold {
  double w[2][N2AR_NZ][N2AR_NH];  // model m: dh_j = sum_k z_k w[m][k][j]
  double h0[2][N2AR_NH];          // pre-activations at all-zero PIPs
  double e0[2][N2AR_NH];          // exp(-h0)
  double c1[2][N2AR_NH];          // h0 (1 - logistic(h0))
  double wo[2][N2AR_NH];          // [0,16): W1[:,0]-W1[:,1] of sub-network 0 (q_N1 - q_N2);
                                  // [16,32): the same for sub-network 1 (q_N1' - q_N2');
                                  // [32,40): W1[:,0] of sub-network 2 (q_Ar)
};

// monomial k of (v0, v1, v2, v3) = (y3, y6, y8, y9): exponents in the order
// degree 1 (v0..v3), degree 2 (vi vj, i <= j), degree 3 (vi vj vl, i <= j <= l)
struct N2arMonomial {
  int deg;
  int v[3];
};
inline N2arMonomial n2ar_monomial(int k) {
  int n = 0;
  for (int deg = 1; deg <= 3; ++deg)
    for (int i = 0; i < 4; ++i)
      for (int j = (deg >= 2 ? i : 0); j < (deg >= 2 ? 4 : 1); ++j)
        for (int l = (deg >= 3 ? j : 0); l < (deg >= 3 ? 4 : 1); ++l) {
          if (n == k) return {deg, {i, deg >= 2 ? j : -1, deg >= 3 ? l : -1}};
          ++n;
        }
  return {0, {-1, -1, -1}};
}

// builds the fold from the generated tables (hh_n2ar_host.cpp); returns 0 on
// success, -1 when a PIP monomial has no Ar pair (the basis is not purified)
int n2ar_build_fold(N2arDipFold *out);

// The PES network in the layout of the trajectory kernels' compact loop: one
// row of 20 (17 used) first-layer weights per hidden unit, so the loop over the
// 32 hidden units reads each row with vector loads from shared memory.
constexpr int N2AR_PES_NP = 17;
constexpr int N2AR_PES_NH = 32;
constexpr int N2AR_PES_ROW = 20;
template <typename T> struct N2arPesNet {
  T w0t[N2AR_PES_NH][N2AR_PES_ROW];  // w0t[j][i] = W0[i][j]
  // the hidden units in pairs: w0p[p][2 i + b] = W0[i][2 p + b], so that (W0[i][2p],
  // W0[i][2p + 1]) is one 8-byte word
  T w0p[N2AR_PES_NH / 2][2 * N2AR_PES_ROW];
  T b0[N2AR_PES_NH];
  T w1[N2AR_PES_NH];
  T xmean[N2AR_PES_ROW];
  T ixscale[N2AR_PES_ROW];           // 1 / xscale
  T ymean, yscale, b1, pad;
};
void n2ar_build_pes(N2arPesNet<double> *d, N2arPesNet<float> *f);
