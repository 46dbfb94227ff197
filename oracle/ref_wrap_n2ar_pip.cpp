// C entry points over the reference's own N2-Ar PIP basis functions (compiled
// where they lie, with the Eigen stand-in of shim/Eigen/Dense).  Test
// infrastructure only: pins the PIP tables of hh_n2ar_tables.h.
#include <Eigen/Dense>

extern "C" void evpoly_2_1_4_purify(double *y, Eigen::Ref<Eigen::RowVectorXd> p);
extern "C" void evpoly_jac_2_1_4_purify(Eigen::Ref<Eigen::MatrixXd> jac, double *y);
extern "C" void evpoly_1_1_2_1_3_purify(double *y, Eigen::Ref<Eigen::RowVectorXd> p);
extern "C" void evpoly_2_1_1_1_3_purify(double *y, Eigen::Ref<Eigen::RowVectorXd> p);
extern "C" void evpoly_2_2_1_3_purify(double *y, Eigen::Ref<Eigen::RowVectorXd> p);

// p[17] from y[3]
extern "C" void ref_n2ar_pes_pip(double *y, double *p) {
  evpoly_2_1_4_purify(y, Eigen::Ref<Eigen::RowVectorXd>(p, 17));
}
// jac[3 x 17], column-major: jac[k + 3 i] = d p_i / d y_k
extern "C" void ref_n2ar_pes_jac(double *y, double *jac) {
  for (int i = 0; i < 51; ++i) jac[i] = 0.0;
  evpoly_jac_2_1_4_purify(Eigen::Ref<Eigen::MatrixXd>(jac, 3, 17), y);
}
// p[308] from y[10], the three bases in the order of the dipole model
extern "C" void ref_n2ar_dip_pip(double *y, double *p) {
  evpoly_1_1_2_1_3_purify(y, Eigen::Ref<Eigen::RowVectorXd>(p, 119));
  evpoly_2_1_1_1_3_purify(y, Eigen::Ref<Eigen::RowVectorXd>(p + 119, 119));
  evpoly_2_2_1_3_purify(y, Eigen::Ref<Eigen::RowVectorXd>(p + 238, 70));
}
