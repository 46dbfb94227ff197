// Host builder of the folded N2-Ar dipole charge models (hh_n2ar_fold.h), in
// FP64 from the generated tables.  Compiled by the host compiler, so the tables
// of hh_n2ar_tables.h are plain constexpr arrays here.
#include <cmath>
#include <cstring>

#include "hh_n2ar_fold.h"
#include "hh_n2ar_tables.h"

namespace {
constexpr double L_N2 = 2.07856749;  // src/constants.h:80
// site-pair index (N1, N2, N1', N2', Ar; pairs i < j) -> varying variable 0..3 or -1
int varying(int pair) {
  switch (pair) {
    case 3: return 0;  // N1-Ar
    case 6: return 1;  // N2-Ar
    case 8: return 2;  // N1'-Ar
    case 9: return 3;  // N2'-Ar
    default: return -1;
  }
}
int monomial_index(int deg, const int *v) {
  for (int k = 0; k < N2AR_NZ; ++k) {
    const N2arMonomial m = n2ar_monomial(k);
    if (m.deg != deg) continue;
    bool eq = true;
    for (int i = 0; i < deg; ++i) eq = eq && (m.v[i] == v[i]);
    if (eq) return k;
  }
  return -1;
}
double logistic(double x) { return 1.0 / (1.0 + std::exp(-x)); }
}  // namespace

void n2ar_build_pes(N2arPesNet<double> *d, N2arPesNet<float> *f) {
  std::memset(d, 0, sizeof *d);
  std::memset(f, 0, sizeof *f);
  for (int j = 0; j < N2AR_PES_NH; ++j) {
    for (int i = 0; i < N2AR_PES_NP; ++i) {
      d->w0t[j][i] = hh_n2ar_pes_w0[i][j];
      d->w0p[j / 2][2 * i + (j & 1)] = hh_n2ar_pes_w0[i][j];
    }
    d->b0[j] = hh_n2ar_pes_b0[j];
    d->w1[j] = hh_n2ar_pes_w1[j];
  }
  for (int i = 0; i < N2AR_PES_NP; ++i) {
    d->xmean[i] = hh_n2ar_pes_xmean[i];
    d->ixscale[i] = 1.0 / hh_n2ar_pes_xscale[i];
  }
  d->ymean = hh_n2ar_pes_y[0];
  d->yscale = hh_n2ar_pes_y[1];
  d->b1 = hh_n2ar_pes_b1[0];
  const double *src = reinterpret_cast<const double *>(d);
  float *dst = reinterpret_cast<float *>(f);
  for (size_t k = 0; k < sizeof *d / sizeof(double); ++k) dst[k] = (float)src[k];
}

int n2ar_build_fold(N2arDipFold *out) {
  std::memset(out, 0, sizeof *out);
  static double M[HH_N2AR_DIP_NPIP][N2AR_NZ];
  for (int m = 0; m < 2; ++m) {
    const double a0 = (m == 0) ? 2.0 : 6.0;
    const double yNN = std::exp(-L_N2 / a0), yNQ = std::exp(-L_N2 / std::sqrt(2.0) / a0);
    // values of the fixed pairs: N1-N2, N1-N1', N1-N2', N2-N1', N2-N2', N1'-N2'
    double yc[10] = {yNN, yNQ, yNQ, 0.0, yNQ, yNQ, 0.0, yNN, 0.0, 0.0};
    std::memset(M, 0, sizeof M);
    for (int t = 0; t < HH_N2AR_DIP_NMONO; ++t) {
      double c = 1.0;
      int v[3], deg = 0;
      for (int j = 0; j < 3; ++j) {
        const int pv = hh_n2ar_dip_var[t][j];
        if (pv < 0) continue;
        const int q = varying(pv);
        if (q < 0) c *= yc[pv];
        else v[deg++] = q;
      }
      if (deg == 0) return -1;
      for (int a = 0; a < deg; ++a)  // sort the variable indices
        for (int b = a + 1; b < deg; ++b)
          if (v[b] < v[a]) { int x = v[a]; v[a] = v[b]; v[b] = x; }
      M[hh_n2ar_dip_poly[t]][monomial_index(deg, v)] += c;
    }
    for (int s = 0; s < 3; ++s) {
      const int nin = hh_n2ar_dip_arch[s][0], nh = hh_n2ar_dip_arch[s][1], no = hh_n2ar_dip_arch[s][2];
      const int p0 = hh_n2ar_dip_pipoff[s], h0 = hh_n2ar_dip_b0off[s];
      const double *W0 = &hh_n2ar_dip_w0[m][hh_n2ar_dip_w0off[s]];
      const double *W1 = &hh_n2ar_dip_w1[m][hh_n2ar_dip_w1off[s]];
      for (int j = 0; j < nh; ++j) {
        double b = hh_n2ar_dip_b0[m][h0 + j];
        for (int i = 0; i < nin; ++i)
          b += (0.0 - hh_n2ar_dip_xmean[m][p0 + i]) / hh_n2ar_dip_xscale[m][p0 + i] * W0[i * nh + j];
        out->h0[m][h0 + j] = b;
        out->e0[m][h0 + j] = std::exp(-b);
        out->c1[m][h0 + j] = b * (1.0 - logistic(b));
        for (int k = 0; k < N2AR_NZ; ++k) {
          double a = 0.0;
          for (int i = 0; i < nin; ++i) a += M[p0 + i][k] / hh_n2ar_dip_xscale[m][p0 + i] * W0[i * nh + j];
          out->w[m][k][h0 + j] = a;
        }
        out->wo[m][h0 + j] = (no == 2) ? W1[j * 2 + 0] - W1[j * 2 + 1] : W1[j];
      }
    }
  }
  return 0;
}
