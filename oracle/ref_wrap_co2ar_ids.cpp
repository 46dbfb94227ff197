/* C entry point around the reference CO2-Ar dipole class
 * (PES-IDS/ai_ids_co2ar.cpp), compiled into oracle/_ref.  Test infrastructure only. */
#include "ai_ids_co2ar.hpp"

static AI_IDS_co2_ar g_ids;
static bool g_init = false;

extern "C" void ref_co2ar_dip_mol(double R, double theta, double d[3]) {
    if (!g_init) { g_ids.init(); g_init = true; }
    g_ids.dipole_vector(R, theta, d);
}
