/* CPU restatement of the reference's GB/SA energy-force hot path
 * (JonnyWideFoot/pd.arcus, src/mmlib) -- TEST ORACLE ONLY.
 *
 * This library is test infrastructure: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it, and only as the checker.  It is
 * never part of the product path.  Its parity against the reference itself
 * is pinned by tests/test_oracle_golden.py, which compares it with outputs
 * of the reference library compiled from source (oracle/Makefile, target
 * "ref") on the same inputs (tests/golden/).
 *
 * Units follow the reference exactly: positions in Angstrom, energies in
 * J/molecule, forces in N, masses in kg, epsilon in sqrt(J), charge in e.
 * Every function names the reference lines it restates.
 */
#ifndef PD_ORACLE_H
#define PD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Forcefield settings, the public members of FF_NonBonded (nonbonded.h:55-126)
 * and FF_GeneralizedBorn_Still (gbff.h:127-133). */
typedef struct {
  double cutoff, inner_cutoff, vdw_cutoff, vdw_inner_cutoff;
  double vdw14, elec14;
  double dielectric;          /* FF_NonBonded::Dielectric (fast2 path)   */
  double diel_solute, diel_solvent;
  double still_cutoff, exp_thresh, diel_offset, born_offset;
  double P1, P2, P3, P4, P5;
  int energy_switch, force_switch, ddd, do_vdw, do_elec, vdwcor;
  double ddd_alpha;
  double vdwcor_density, vdwcor_eps, vdwcor_radius, vdwcor_cutoff;
} pdo_params;

/* Physical constants as the reference defines them (forcefield.cpp:18-38). */
void pdo_constants(double out[8]); /* kcal2J J2kcal Na kB Angstrom econv econv_joule halfeconv */

/* BondOrder::reinit (workspace/bondorder.cpp:77-195).  cov lists are CSR
 * (ptr[n+1], idx).  band must hold mid*(n-1) bytes; returns mid, or -1 if
 * band_cap is too small.  Off-diagonal entries are written as triples
 * (i, j, order) in the reference's storage order; *n_off receives their
 * count (off_cap triples at most). */
int pdo_bondorder(int n, const int *ir, const int *c12p, const int *c12i,
                  const int *c13p, const int *c13i, const int *c14p,
                  const int *c14i, int8_t *band, long band_cap, int *off,
                  int off_cap, int *n_off);

/* NeighbourList::calcNewList_InfiniteSpace + correctOffDiagonalBondOrders
 * (workspace/neighbourlist.cpp:162-316).  Writes the packed reference
 * entries (j | bo<<24) per atom in ascending j; ptr has n+1 entries.
 * Returns the entry count, or -1 if cap is exceeded. */
long pdo_nlist(int n, const double *pos, double cutoff, double padding,
               int shadow, int mid, const int8_t *band, int n_off,
               const int *off, int *ptr, int *data, long cap);

/* FF_GeneralizedBorn_Still::calcFixedBornRadiiTerms (gbff.cpp:307-381). */
void pdo_gb_fixed_terms(int n, const double *gbr, const int *c12p,
                        const int *c12i, const double *c12d, const int *c13p,
                        const int *c13i, const double *c13d,
                        const pdo_params *p, double *vj, double *terms123);

/* calcBornRadii_PairwiseApprox (gbff.cpp:415-466). */
void pdo_born_radii(int n, const double *pos, const int *ptr, const int *data,
                    const double *gbr, const double *vj,
                    const double *terms123, const pdo_params *p,
                    double *born);

/* calcForcesIncludingVacuo (gbff.cpp:1449-1818): adds forces (N) to f,
 * writes ene[0..5] = epot, epot_vdw, epot_elec, epot_pol, epot_pol_cross,
 * epot_pol_self (J), per-atom epot (may be NULL) and deda (may be NULL). */
void pdo_gb_forces(int n, const double *pos, const int *ptr, const int *data,
                   const double *q, const double *radius, const double *eps,
                   const double *gbr, const double *vj, const double *born,
                   const pdo_params *p, double *f, double *ene,
                   double *atom_epot, double *deda);

/* calcBornEnergy (gbff.cpp:520-579): returns the Born energy (J);
 * pol[0..2] = epot_pol, epot_pol_cross, epot_pol_self. */
double pdo_born_energy(int n, const double *pos, const int *ptr,
                       const int *data, const double *q, const double *born,
                       const pdo_params *p, double *pol);

/* FF_NonBonded_CalcForces_T_fast2 (nonbonded.cpp:548-893), infinite space.
 * Adds forces (N) to f; ene[0..3] = epot, epot_vdw, epot_elec,
 * InternalVirial (J). */
void pdo_nonbonded(int n, const double *pos, const int *ptr, const int *data,
                   const double *q, const double *radius, const double *eps,
                   const pdo_params *p, double *f, double *ene);

/* FF_Bonded::calcForces (ffbonded.cpp:809-823, 885-940, 994-1129,
 * 1207-1499, 1534-1559).  Adds forces (N) to f; ene[0..4] = epot_bond,
 * epot_angle, epot_torsion (torsions+impropers), InternalVirial, epot. */
void pdo_bonded(int n, const double *pos, int nb, const int *bij,
                const double *blk, int na, const int *aiaj, const double *akt,
                int nt, const int *tidx, const int *tterms,
                const double *tpar, int ni, const int *iidx,
                const int *iterms, const double *ipar, double *f,
                double *ene);

/* MolecularDynamics integrator steps (protocols/md.cpp).  x in Angstrom,
 * v in m/s, f in N, mass in kg; normals[6n] in the order the reference's
 * three nrand() pairs produce them per atom (n1x n2y n2x n1z n1y n2z).
 * step/steps are the protocol's Step and Steps.  Returns ekin (J). */
double pdo_langevin_step(int n, double *x, double *v, const double *f,
                         const double *mass, const double *normals, double dt,
                         double gamma, double temp, int step, int steps);
double pdo_velocity_verlet_step(int n, double *x, double *v, const double *f,
                                const double *mass, double dt);
double pdo_beeman_step(int n, double *x, double *v, const double *f,
                       double *fold, const double *mass, double dt, int step,
                       int steps);

/* FF_SASA_LCPO (forcefields/lcpo.cpp) over the reference's neighbour list
 * (ptr/data as pdo_nlist writes them: entries j | bo << 24, ascending j;
 * only the j < i part of each row is read, lcpo.cpp:446-447).
 * radius: LCPO type radius + 1.4 (A); p: P1..P4 per atom ([n][4]); sigma:
 * the atomic solvation parameter per atom (J/A^2 as the reference forms it
 * from GlobalASP, or any other unit: the results scale with it); use: 0
 * for the atoms the component ignores.
 * energy_only = 0: calcLCPOSasaForces(true) (lcpo.cpp:623-946): writes
 *   sasa[n] (A^2) and deriv[3n] (SASAderiv: sigma units per A, the
 *   force direction) and returns epot_cav = the sum of sasa * sigma.
 * energy_only = 1: calcLCPOSasaEnergies(true) (lcpo.cpp:414-566): writes
 *   sasa and returns epot_cav; deriv is not touched (may be NULL).
 * The overlap lists hold at most 80 partners per atom (lcpo.h Nlistmax);
 * *truncated (may be NULL) receives how many partners did not fit. */
double pdo_lcpo(int n, const double *pos, const int *ptr, const int *data,
                const double *radius, const double *p, const double *sigma,
                const int8_t *use, int energy_only, double *sasa,
                double *deriv, long *truncated);

#ifdef __cplusplus
}
#endif
#endif
