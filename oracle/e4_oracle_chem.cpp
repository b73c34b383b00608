/*
 * e4_oracle_chem.cpp -- thermally perfect gas and finite-rate chemistry of the
 * CPU FP64 oracle.  TEST INFRASTRUCTURE ONLY (see e4_oracle.cpp).
 */
#include "e4_oracle_internal.h"

namespace e4o {

void GasModel::init_therm_perf_air5() { kind = E4O_GAS_THERM_PERF_5SP_AIR; nsp = 5; }
bool GasModel::tp_update_thermo_from_pT(GasState&) const { return false; }
bool GasModel::tp_update_thermo_from_rhou(GasState&) const { return false; }
bool GasModel::tp_update_thermo_from_rhoT(GasState&) const { return false; }
bool GasModel::tp_update_sound_speed(GasState&) const { return false; }
int Sim::chemistry_step(double) { return E4O_ERR_CHEM; }

}  // namespace e4o
