// CH4-CO2 dipole table folded for the batched dipole kernel (hh_ch4co2_dip.cuh),
// built on the host by hh_ch4co2_host.cpp from the generated tables.
#pragma once
#include <vector>

struct Ch4Co2FoldHost {
  int n_entry = 0, n_group = 0;
  std::vector<double> coef;             // [NSEG][n_entry][4]: cubic in R - centre of each piece
  std::vector<unsigned char> y2;        // [n_entry]: Y2 index (m2-major, even l2, cos then sin)
  std::vector<unsigned int> grp;        // [n_group]: cs | comp << 1 | entries << 3
  std::vector<unsigned short> gcount;   // [(l1, m1), m1-major]: groups at that Y1
  // the same stream with every group padded to whole batches of 4 entries (zero
  // coefficients), for the batched kernel loop
  int n_batch = 0;
  std::vector<double> bcoef;            // [NSEG][4 n_batch][4]
  std::vector<unsigned char> by2;       // [4 n_batch]
  std::vector<unsigned int> bmeta;      // [n_batch]: cs | comp << 1 | (last batch of its group) << 3 | lm << 8
};

// entries e = (component, Y1, Y2) with K_e(R) = sum over the reference's terms of
// coef * rad_b(R) * N(l1, m1) * N(l2, m2), N(l, m) = sqrt((l+m)!/(l-m)!) (the kernel's
// harmonics carry sqrt((l-m)!/(l+m)!)); returns 0, or -1 on an unexpected table
int ch4co2_build_fold(Ch4Co2FoldHost *out);

// coefficient images of the tensor-core dipole kernel (hh_ch4co2_tc.cuh): per radial
// piece, pass and K-chunk the TF32 (hi, lo) split of B_c[Y1 column, 4 Y2 + power] in
// the layout of hh_ch4co2_tc_layout.h; blob holds NSEG * CH4TC_PIECE_BYTES / 4 floats.
// Returns 0, or -1 on an unexpected table.
int ch4co2_build_tc_blob(const Ch4Co2FoldHost &f, std::vector<float> *blob);
