// Entry points into the reference's CH4-CO2 dipole, compiled from its own sources
// (PES-IDS/ai_ids_ch4_co2.cpp, PES-IDS/ai_ids_ch4_co2_lib.cpp, src/angles_handler.cpp)
// into oracle/_ref/libref_ch4co2_ids.so.  Test infrastructure only.
#include "ai_ids_ch4_co2.hpp"
#include "angles_handler.hpp"

extern "C" void dipole_lab(double *qlab, double diplab[3]);

extern "C" {
void ref_ch4co2_init(void) { dipole_init(); }
void ref_ch4co2_dipole_vector(const double *qkal, double d[3]) { dipole_vector((double *)qkal, d); }
void ref_ch4co2_lab_to_kal(const double *qlab, double *qkal) {
  CH4_linear_molecule_lab_to_kal((double *)qlab, qkal);
}
void ref_ch4co2_dipole_lab(const double *qlab, double d[3]) { dipole_lab((double *)qlab, d); }
}
