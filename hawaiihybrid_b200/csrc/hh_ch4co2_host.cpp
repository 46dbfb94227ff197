// Host builder of the folded CH4-CO2 dipole table (hh_ch4co2_fold.h) from the
// expanded reference tables of hh_ch4co2_tables.h, in FP64.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <tuple>

#include "hh_ch4co2_fold.h"
#include "hh_ch4co2_tables.h"
#include "hh_ch4co2_tc_layout.h"

namespace {
void lm_of(int code, int *l, int *m, int *cs) {
  const int i = code >> 1;
  int L = 0;
  while ((L + 1) * (L + 2) / 2 <= i) ++L;
  *l = L;
  *m = i - L * (L + 1) / 2;
  *cs = code & 1;
}
// nearest TF32 value (10 explicit mantissa bits, ties away from zero) of a float
float tf32_rna(float v) {
  uint32_t b;
  memcpy(&b, &v, 4);
  b = (b + 0x1000u) & ~0x1FFFu;
  float r;
  memcpy(&r, &b, 4);
  return r;
}
double norm_lm(int l, int m) {  // sqrt((l+m)! / (l-m)!)
  double p = 1.0;
  for (int k = l - m + 1; k <= l + m; ++k) p *= k;
  return std::sqrt(p);
}
}  // namespace

int ch4co2_build_fold(Ch4Co2FoldHost *out) {
  // Y2 index in the kernel's generation order
  std::map<std::tuple<int, int, int>, int> y2idx;
  int n2 = 0;
  for (int m = 0; m <= HH_CH4CO2_L2MAX; ++m)
    for (int l = m; l <= HH_CH4CO2_L2MAX; ++l)
      if ((l & 1) == 0) {
        y2idx[{l, m, 0}] = n2++;
        if (m > 0) y2idx[{l, m, 1}] = n2++;
      }
  // entries keyed in the kernel's loop order: m1, l1, cs1, component, Y2
  using Key = std::tuple<int, int, int, int, int>;
  std::map<Key, std::vector<double>> acc;
  for (int t = 0; t < HH_CH4CO2_NTERM; ++t) {
    const short *ix = hh_ch4co2_tidx[t];
    int l1, m1, c1, l2, m2, c2;
    lm_of(ix[2], &l1, &m1, &c1);
    lm_of(ix[3], &l2, &m2, &c2);
    if (l1 > HH_CH4CO2_L1MAX) return -1;
    auto it = y2idx.find({l2, m2, c2});
    if (it == y2idx.end()) return -1;
    std::vector<double> &k = acc[Key(m1, l1, c1, ix[1], it->second)];
    if (k.empty()) k.assign(HH_CH4CO2_NSEG * 4, 0.0);
    const double w = hh_ch4co2_tcoef[t] * norm_lm(l1, m1) * norm_lm(l2, m2);
    for (int s = 0; s < HH_CH4CO2_NSEG; ++s)
      for (int j = 0; j < 4; ++j) k[s * 4 + j] += w * hh_ch4co2_rad[ix[0]][s][j];
  }
  const int E = (int)acc.size();
  out->n_entry = E;
  out->coef.assign((size_t)HH_CH4CO2_NSEG * E * 4, 0.0);
  out->y2.assign(E, 0);
  out->grp.clear();
  out->gcount.assign((HH_CH4CO2_L1MAX + 1) * (HH_CH4CO2_L1MAX + 2) / 2, 0);
  // (l1, m1) -> position in the m1-major order of the kernel
  auto lm_pos = [](int l, int m) {
    int p = 0;
    for (int mm = 0; mm < m; ++mm) p += HH_CH4CO2_L1MAX + 1 - mm;
    return p + (l - m);
  };
  int e = 0;
  Key prev(-1, -1, -1, -1, -1);
  for (auto &kv : acc) {
    const Key &k = kv.first;
    const bool same = std::get<0>(k) == std::get<0>(prev) && std::get<1>(k) == std::get<1>(prev) &&
                      std::get<2>(k) == std::get<2>(prev) && std::get<3>(k) == std::get<3>(prev);
    if (!same) {
      out->grp.push_back((unsigned)std::get<2>(k) | ((unsigned)std::get<3>(k) << 1));
      out->gcount[lm_pos(std::get<1>(k), std::get<0>(k))]++;
    }
    out->grp.back() += 1u << 3;
    out->y2[e] = (unsigned char)std::get<4>(k);
    for (int s = 0; s < HH_CH4CO2_NSEG; ++s)
      for (int j = 0; j < 4; ++j) out->coef[((size_t)s * E + e) * 4 + j] = kv.second[s * 4 + j];
    prev = k;
    ++e;
  }
  out->n_group = (int)out->grp.size();
  // padded batches: each group's entries followed by zero entries up to a multiple of 4
  out->bcoef.clear();
  out->by2.clear();
  out->bmeta.clear();
  std::vector<int> order;  // entry index or -1 (padding), in batch order
  {
    int g = 0, lm = 0, e0 = 0;
    for (int m = 0; m <= HH_CH4CO2_L1MAX; ++m)
      for (int l = m; l <= HH_CH4CO2_L1MAX; ++l, ++lm)
        for (int k = 0; k < out->gcount[lm]; ++k, ++g) {
          const unsigned d = out->grp[g];
          const int cnt = int(d >> 3);
          const int nb = (cnt + 3) / 4;
          for (int b = 0; b < nb; ++b) {
            for (int j = 0; j < 4; ++j) order.push_back(4 * b + j < cnt ? e0 + 4 * b + j : -1);
            out->bmeta.push_back((d & 7u) | (b == nb - 1 ? 8u : 0u) | ((unsigned)lm << 8));
          }
          e0 += cnt;
        }
  }
  out->n_batch = (int)out->bmeta.size();
  const size_t EP = order.size();
  out->bcoef.assign((size_t)HH_CH4CO2_NSEG * EP * 4, 0.0);
  out->by2.assign(EP, 0);
  for (size_t i = 0; i < EP; ++i) {
    if (order[i] < 0) continue;
    out->by2[i] = out->y2[order[i]];
    for (int s = 0; s < HH_CH4CO2_NSEG; ++s)
      for (int j = 0; j < 4; ++j)
        out->bcoef[((size_t)s * EP + i) * 4 + j] = out->coef[((size_t)s * E + order[i]) * 4 + j];
  }
  return 0;
}

int ch4co2_build_tc_blob(const Ch4Co2FoldHost &f, std::vector<float> *blob) {
  using namespace hh;
  const int E = f.n_entry;
  // B[piece][component][column][K] in FP64 from the entry stream (groups in (m1, l1, cs,
  // component) order, gcount groups per (l1, m1) in m-major order)
  const size_t per_comp = (size_t)CH4TC_N * CH4TC_K;
  std::vector<double> B((size_t)HH_CH4CO2_NSEG * 3 * per_comp, 0.0);
  int g = 0, e = 0, lm = 0;
  for (int m = 0; m <= HH_CH4CO2_L1MAX; ++m)
    for (int l = m; l <= HH_CH4CO2_L1MAX; ++l, ++lm)
      for (int k = 0; k < f.gcount[lm]; ++k, ++g) {
        const unsigned d = f.grp[g];
        const int cs = int(d & 1u), comp = int((d >> 1) & 3u), cnt = int(d >> 3);
        if (comp > 2 || (m == 0 && cs == 1)) return -1;
        const int col = ch4tc_y1_col(l, m, cs, HH_CH4CO2_L1MAX);
        if (col >= CH4TC_NY1) return -1;
        for (int i = 0; i < cnt; ++i, ++e) {
          const int y2 = f.y2[e];
          for (int s = 0; s < HH_CH4CO2_NSEG; ++s)
            for (int j = 0; j < 4; ++j)
              B[((size_t)s * 3 + comp) * per_comp + (size_t)col * CH4TC_K + 4 * y2 + j] =
                  f.coef[((size_t)s * E + e) * 4 + j];
        }
      }
  if (e != E) return -1;
  blob->assign((size_t)HH_CH4CO2_NSEG * CH4TC_PIECE_BYTES / 4, 0.0f);
  for (int s = 0; s < HH_CH4CO2_NSEG; ++s)
    for (int q = 0; q < 2; ++q) {
      const int ncomp = q == 0 ? 2 : 1, img = (q == 0 ? CH4TC_IMG0 : CH4TC_IMG1) / 4;
      for (int c = 0; c < CH4TC_NCHUNK; ++c) {
        float *hi = blob->data() + ch4tc_blob_off(s, q, c) / 4, *lo = hi + img;
        for (int cc = 0; cc < ncomp; ++cc) {
          const int comp = q == 0 ? cc : 2;
          for (int n = 0; n < CH4TC_N; ++n)
            for (int kk = 0; kk < CH4TC_KC; ++kk) {
              // the chunk's column kk: power kk % 4 of the Y2 its group holds
              const int k = ch4tc_k_of(c, kk / 4);
              const double v = k < 0 ? 0.0 : B[((size_t)s * 3 + comp) * per_comp + (size_t)n * CH4TC_K + 4 * k + kk % 4];
              const float h = tf32_rna((float)v);
              const int off = ch4tc_img_off(cc * CH4TC_N + n, kk);
              hi[off] = h;
              lo[off] = tf32_rna((float)(v - (double)h));
            }
        }
      }
    }
  return 0;
}
