/*
 * surface_scatter_defined.cpp -- ORACLE TEST INFRASTRUCTURE.
 *
 * Replaces src/ParSurfaceScatter.cpp (whole file, 193 lines) in the oracle
 * build.  That file reads the local `drand` uninitialised in
 * HoleSurfacePhononScatter (src/ParSurfaceScatter.cpp:72,94) and in
 * ElectronSurfacePhononScatter (:124,149), so the reference's mechanism
 * choice there is undefined behaviour.  The B200 engine and this oracle both
 * define it as one draw scaled by the sum of the per-mechanism rates at the
 * particle's energy:  drand = Random() * sum_i sca[i]  (sum in index order).
 * Everything else below follows the reference line for line:
 *   GetSurfScRate            src/ParSurfaceScatter.cpp:3-45  (the debug dump
 *                            under Flag_calSurfscatt, :24-44, is left out)
 *   ParticleSurfaceScatter   :48-61
 *   HoleSurfacePhononScatter :64-114
 *   ElectronSurfacePhononScatter :117-192
 */
#include "mcmodel.h"

void MeshQuantities::GetSurfScRate() {
  double *roughnessRate, *surfPhononRate;
  if (par_type == PELEC) {
    c_e_roughnessRate->ExtractView(&roughnessRate);
    c_e_surfPhononRate->ExtractView(&surfPhononRate);
  } else {
    c_h_roughnessRate->ExtractView(&roughnessRate);
    c_h_surfPhononRate->ExtractView(&surfPhononRate);
  }
  SurfRoughnessScRate = roughnessRate[C_LINDEX_GHOST_ONE(icell, jcell, kcell)];
  SurfPhononScRate = surfPhononRate[C_LINDEX_GHOST_ONE(icell, jcell, kcell)];
  SurfScGamma = SurfRoughnessScRate + SurfPhononScRate;
}

void MeshQuantities::ParticleSurfaceScatter() {
  if (Random() * SurfScGamma < SurfRoughnessScRate) {
    idir = SurfaceDir[(*c_nearestSurf)[C_LINDEX_GHOST_ONE(icell, jcell, kcell)]];
    Diffuse();
  } else {
    if (par_type == PELEC)
      ElectronSurfacePhononScatter();
    else if (par_type == PHOLE)
      HoleSurfacePhononScatter();
  }
}

void MeshQuantities::HoleSurfacePhononScatter() {
  int iscat;
  double drand, dscat, total;
  double sca[MNScaHole * NBH];
  Flag_SelfScatter = false;
  band.CALSCATTH(energy, sca, iband);
  total = 0.0;
  for (int i = 0; i < band.scprh * band.nband[PHOLE]; ++i) total += sca[i];
  drand = Random() * total;
  iscat = -1;
  dscat = 0.0;
  while (drand > dscat) {
    iscat = iscat + 1;
    if (iscat >= (band.scprh * band.nband[PHOLE])) {
      Flag_SelfScatter = true;
      break;
    }
    dscat = dscat + sca[iscat];
  }
  if (!Flag_SelfScatter) {
    if (((iscat % band.scprh) + 1) == band.scprh)
      HSCATII(iscat);
    else
      HPSCAT(iscat);
  }
}

void MeshQuantities::ElectronSurfacePhononScatter() {
  int iscat;
  double drand, dscat, total;
  double sca[MNScaEle * NBE];
  Flag_SelfScatter = false;
  band.CALSCATTE(energy, sca, iband);
  total = 0.0;
  for (int i = 0; i < band.scpre * band.nband[PELEC]; ++i) total += sca[i];
  drand = Random() * total;
  iscat = -1;
  dscat = 0.0;
  while (drand > dscat) {
    iscat = iscat + 1;
    if (iscat >= (band.scpre * band.nband[PELEC])) {
      Flag_SelfScatter = true;
      break;
    }
    dscat = dscat + sca[iscat];
  }
  if (!Flag_SelfScatter) {
    if (((iscat % band.scpre) + 1) == band.scpre)
      ESCATII(iscat);
    else
      EPSCAT(iscat);
  }
}
