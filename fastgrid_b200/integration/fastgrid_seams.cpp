// FastGrid's two map-calculation seams, implemented on the B200 engine.
//
// This is the binding a FastGrid maintainer adds to switch FastGrid's own
// driver (fastgrid/main.cpp, programMain) to the GPU engine: the translation
// unit replaces the bodies of
//
//   calculateElectrostaticMapAsync / synchronizeCalculation
//       (electrostatics/Electrostatics.h:32-36; CPU body electrostatics/Cpu.cpp:90-127)
//   calculateGridmaps
//       (CalculateGridmaps.h:30-31; body CalculateGridmaps.cpp:433-485)
//
// and everything else — the GPF/PDBQT loader, the parameter library, the
// pair-energy and desolvation tables, the bond vectors, the covalent maps, the
// floating grid and the .map/.fld/.xyz writers — stays FastGrid's own code.
// oracle/Makefile (target `seams`) compiles FastGrid's sources without those
// two bodies plus this file, linked to libfastgrid_b200.so.
//
// Both seams hand FastGrid's arrays to the engine's C ABI (include/
// fastgrid_b200.h) and store the FP32 results in FastGrid's FP64 map arrays
// rounded exactly as FastGrid rounds them (roundOutput, autogrid.h:128-131).
#include <cstdio>
#include <vector>

#include "CalculateGridmaps.h"
#include "Exceptions.h"
#include "Utils.h"
#include "autogrid.h"
#include "electrostatics/Electrostatics.h"
#include "fastgrid_b200.h"

namespace {

// One engine context for the process, on the device --cuda-dev names.
ag_ctx* engine(const ProgramParameters& programParams) {
  static ag_ctx* ctx = nullptr;
  if (!ctx && ag_ctx_create(programParams.getDeviceIDCUDA(), &ctx) != AG_OK) {
    fprintf(stderr, "%s: ERROR: %s\n", programParams.getProgramName(), ag_last_error());
    throw ExitProgram(-2);
  }
  return ctx;
}

void check(int rc, const ProgramParameters& programParams) {
  if (rc != AG_OK) {
    fprintf(stderr, "%s: ERROR: %s\n", programParams.getProgramName(), ag_last_error());
    throw ExitProgram(-2);
  }
}

ag_grid gridOf(const InputData* input) {
  ag_grid g;
  g.nx = input->numGridPoints.x;
  g.ny = input->numGridPoints.y;
  g.nz = input->numGridPoints.z;
  g.spacing = input->gridSpacing;
  return g;
}

}  // namespace

void* calculateElectrostaticMapAsync(const InputData* input, const ProgramParameters& programParams,
                                     GridMapList& gridmaps) {
  Timer* t = programParams.benchmarkEnabled() ? Timer::startNew("Electrostatic map      ") : 0;
  const int n = input->numReceptorAtoms;
  std::vector<double> xyzw(4 * (size_t)n);
  for (int i = 0; i < n; i++) {
    xyzw[4 * (size_t)i + 0] = input->receptorAtom[i].x;
    xyzw[4 * (size_t)i + 1] = input->receptorAtom[i].y;
    xyzw[4 * (size_t)i + 2] = input->receptorAtom[i].z;
    xyzw[4 * (size_t)i + 3] = input->receptorAtom[i].w;  // q * coeff_estat (* 1/diel for the constant dielectric)
  }
  const ag_grid g = gridOf(input);
  std::vector<float> out((size_t)input->numGridPointsPerMap);
  check(ag_emap(engine(programParams), &g, n, xyzw.data(), input->distDepDiel ? input->epsilon : nullptr, out.data()),
        programParams);
  double* e = gridmaps.getElectrostaticMap().energies;
  for (size_t p = 0; p < out.size(); p++) e[p] = roundOutput((double)out[p]);
  if (t) t->stopAndLog(stderr);
  gridmaps.saveElectrostaticMap();
  return 0;  // computed synchronously: the handle is empty
}

void synchronizeCalculation(void*) {}

void calculateGridmaps(const InputData* input, const ProgramParameters& programParams, GridMapList& gridmaps,
                       const ParameterLibrary& parameterLibrary, const PairwiseInteractionEnergies& energyLookup,
                       const DesolvExpFunc& desolvExpFunc, const BondVectors* bondVectors) {
  Timer* t = programParams.benchmarkEnabled() ? Timer::startNew("Atom & desolvation maps") : 0;
  const int n = input->numReceptorAtoms;
  const int nmaps = gridmaps.getNumAtomMaps();
  const int ntypes = input->numReceptorTypes > 0 ? input->numReceptorTypes : 1;
  const size_t np = (size_t)input->numGridPointsPerMap;

  // Receptor (InputData.h:53-58 + BondVectors.h:31-34) as the engine's structure of arrays.
  std::vector<double> xyzw(4 * (size_t)n), rv(3 * (size_t)n), rv2(3 * (size_t)n);
  std::vector<int> hbond(n);
  std::vector<unsigned char> disorder(n);
  for (int i = 0; i < n; i++) {
    xyzw[4 * (size_t)i + 0] = input->receptorAtom[i].x;
    xyzw[4 * (size_t)i + 1] = input->receptorAtom[i].y;
    xyzw[4 * (size_t)i + 2] = input->receptorAtom[i].z;
    xyzw[4 * (size_t)i + 3] = input->receptorAtom[i].w;
    hbond[i] = (int)input->hbond[i];
    disorder[i] = bondVectors->disorder[i] ? 1 : 0;
    rv[3 * (size_t)i + 0] = bondVectors->rvector[i].x;
    rv[3 * (size_t)i + 1] = bondVectors->rvector[i].y;
    rv[3 * (size_t)i + 2] = bondVectors->rvector[i].z;
    rv2[3 * (size_t)i + 0] = bondVectors->rvector2[i].x;
    rv2[3 * (size_t)i + 1] = bondVectors->rvector2[i].y;
    rv2[3 * (size_t)i + 2] = bondVectors->rvector2[i].z;
  }
  ag_receptor rec;
  rec.n_atoms = n;
  rec.xyzw = xyzw.data();
  rec.charge = input->charge;
  rec.vol = input->vol;
  rec.solpar = input->solpar;
  rec.type = input->atomType;
  rec.hbond = hbond.data();
  rec.disorder = disorder.data();
  rec.rexp = bondVectors->rexp;
  rec.rvector = rv.data();
  rec.rvector2 = rv2.data();

  // Tables (PairwiseInteractionEnergies.h:42-45, DesolvExpFunc.h:33-36) and per-map parameters (GridMap.h:27-57).
  std::vector<double> energy((size_t)ntypes * AG_TABLE_LEN * (nmaps > 0 ? nmaps : 1)), sol(AG_TABLE_LEN);
  for (int a = 0; a < ntypes; a++)
    for (int i = 0; i < AG_TABLE_LEN; i++)
      for (int m = 0; m < nmaps; m++) energy[((size_t)a * AG_TABLE_LEN + i) * nmaps + m] = energyLookup(a, i, m);
  for (int i = 0; i < AG_TABLE_LEN; i++) sol[i] = desolvExpFunc(i);
  std::vector<int> mapHbond(nmaps), mapIsHB(nmaps), mapCov(nmaps);
  std::vector<double> solparProbe(nmaps), volProbe(nmaps);
  for (int m = 0; m < nmaps; m++) {
    mapHbond[m] = (int)gridmaps[m].hbond;
    mapIsHB[m] = gridmaps[m].isHBonder;
    mapCov[m] = gridmaps[m].isCovalent ? 1 : 0;
    solparProbe[m] = gridmaps[m].solparProbe;
    volProbe[m] = gridmaps[m].volProbe;
  }
  ag_affinity_params par;
  par.n_maps = nmaps;
  par.n_types = ntypes;
  par.energy = energy.data();
  par.sol = sol.data();
  par.map_hbond = mapHbond.data();
  par.map_is_hbonder = mapIsHB.data();
  par.map_is_covalent = mapCov.data();
  par.solpar_probe = solparProbe.data();
  par.vol_probe = volProbe.data();
  par.solpar_q = input->solparQ;
  par.hydrogen = parameterLibrary.getAtomParameterRecIndex("HD");

  const ag_grid g = gridOf(input);
  std::vector<float> maps(np * (nmaps > 0 ? nmaps : 1)), dmap(np);
  check(ag_affinity(engine(programParams), &g, &rec, &par, maps.data(), dmap.data()), programParams);

  // Every atom map is rounded at the end of the reference's per-point loop
  // (CalculateGridmaps.cpp:307-315), covalent ones included (their values
  // come from initCovalentMaps).
  for (int m = 0; m < nmaps; m++) {
    double* e = gridmaps[m].energies;
    if (gridmaps[m].isCovalent)
      for (size_t p = 0; p < np; p++) e[p] = roundOutput(e[p]);
    else
      for (size_t p = 0; p < np; p++) e[p] = roundOutput((double)maps[(size_t)m * np + p]);
  }
  double* d = gridmaps.getDesolvationMap().energies;
  for (size_t p = 0; p < np; p++) d[p] = roundOutput((double)dmap[p]);
  if (t) t->stopAndLog(stderr);
}
