/*
 * Oracle for the grid-map path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64 restatement of FastGrid's CPU map calculation, used by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
 * checker.  It is never linked into, loaded by, or called from the product
 * library (fastgrid_b200/), which has no CPU fallback.
 *
 * Pinning: with the reference's rounding (oracle_round) applied, these
 * functions reproduce the reference's golden maps value-for-value:
 * tests/original_win32/colagen2.{C,HD,OA,e,d}.map and
 * AG421/Tests/py_hsg1_sm.{A,C,HD,N,NA,OA,e,d}.map, and the maps FastGrid's
 * own CPU build (oracle/_ref/fastgrid4) writes for seeded synthetic receptors
 * (tests/test_oracle.py, fixtures in tests/golden/).
 */
#ifndef AG_ORACLE_H
#define AG_ORACLE_H
#include "../include/fastgrid_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Electrostatic map over every grid point (Cpu.cpp:27-88).  ddd = 1 selects
 * the tabulated distance-dependent dielectric, 0 the constant one. */
void oracle_emap(const ag_grid* g, int n_atoms, const double* xyzw, const double* inv_eps, int ddd, double* out);
/* The same for a list of flat point indices. */
void oracle_emap_points(const ag_grid* g, int n_atoms, const double* xyzw, const double* inv_eps, int ddd,
                        int n_points, const int64_t* idx, double* out);

/* Affinity maps + d-map for every grid point, brute force over all atoms in
 * file order (CalculateGridmaps.cpp:238-316 with findClosestHBond :65-82).
 * out_maps: [n_maps][n_points]; covalent maps are left at 0. */
void oracle_affinity(const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p, double* out_maps,
                     double* out_dmap);
/* The same for a list of flat point indices, using a cell list to find the
 * atoms within 8 A (summed in file order, like the reference's cutoff grid). */
void oracle_affinity_points(const ag_grid* g, const ag_receptor* r, const ag_affinity_params* p, int n_points,
                            const int64_t* idx, double* out_maps, double* out_dmap);

/* Restated lookup tables (InputDataLoader.cpp:723-724, DesolvExpFunc.cpp:27-43,
 * PairwiseInteractionEnergies.cpp:85-115). */
void oracle_ddd_table(double* eps8192);
void oracle_sol_table(double coeff_desolv, double* sol8192);
void oracle_pair_table(int xA, int xB, double Rij, double epsij, double r_smooth, double* out8192);

/* roundOutput (autogrid.h:255-258). */
double oracle_round(double a);

#ifdef __cplusplus
}
#endif
#endif
