/* pdgpu: B200 (sm_100a) GB/SA energy-force hot path of PD (JonnyWideFoot/pd.arcus).
 *
 * C ABI of libpdgpu.so.  Plain pointers and sizes only.  Every entry point
 * returns PDGPU_OK (0) or a negative status; pdgpu_last_error() gives the
 * message of the last failure on the calling thread.  Inputs and outputs
 * use the reference's own units: positions in Angstrom, energies in
 * J/molecule, forces in N, masses in kg, LJ epsilon in sqrt(J), LJ radius
 * (half Rmin) and GB radius in Angstrom, charges in e.
 *
 * Each entry point names the reference interface it replaces
 * (paths relative to the reference's src/mmlib).
 *
 * Threading: a context is used by one host thread at a time; calls on one
 * context are serialised on its CUDA stream.  Separate contexts may be
 * driven from separate threads.
 */
#ifndef PDGPU_H
#define PDGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define PDGPU_OK 0
#define PDGPU_ERR_ARG -1        /* bad argument (ArgumentException)           */
#define PDGPU_ERR_CUDA -2       /* CUDA runtime failure                        */
#define PDGPU_ERR_NOMEM -3      /* device allocation failed (OutOfMemory)      */
#define PDGPU_ERR_UNSTABLE -4   /* NaN energy (ProcedureException "unstable") */
#define PDGPU_ERR_STATE -5      /* call out of order (e.g. no neighbour list)  */
#define PDGPU_ERR_BUDGET -6     /* admission refused: HBM budget exhausted     */
#define PDGPU_ERR_NODEVICE -7   /* no CUDA device / extension not usable       */

typedef struct pdgpu_ctx pdgpu_ctx;

/* ------------------------------------------------------------------ settings
 * Public members of FF_NonBonded (forcefields/nonbonded.h:55-126) and
 * FF_GeneralizedBorn_Still (forcefields/gbff.h:127-133), same names and
 * meaning.  pdgpu_ff_params_default() fills the values a freshly constructed
 * FF_GeneralizedBorn_Still carries (gbff.cpp:17-38, nonbonded.cpp:968-1004). */
typedef struct {
  double Cutoff, InnerCutoff, VdwCutoff, VdwInnerCutoff;
  double Vdw14Scaling, Elec14Scaling;
  double Dielectric;           /* FF_NonBonded::Dielectric (stand-alone LJ/Coulomb) */
  double DielectricSolute, DielectricSolvent;
  double GbsaStillCutoff, ExpApproxThreshold, DielectricOffset, BornRadiusOffset;
  double P1, P2, P3, P4, P5;   /* Still parameters (SOLVATION_GENERALISED_BORN)     */
  double DDDielectricAlpha;
  double VdwCorDensity, VdwCorEpsilon, VdwCorRadius, VdwCorCutoff;
  double Padding;              /* NeighbourListBase::Padding (neighbourlist.cpp:18) */
  int32_t FastMode, EnergySwitch, ForceSwitch, DDDielectric, DoVdw, DoElec, VdwCor;
  int32_t _reserved;
} pdgpu_ff_params;

void pdgpu_ff_params_default(pdgpu_ff_params *p);

/* ------------------------------------------------------------------ context */
/* Replaces: nothing in the reference (it is host-only); owns the device,
 * one CUDA stream and the resident systems. */
int pdgpu_ctx_create(int device, pdgpu_ctx **out);
int pdgpu_ctx_destroy(pdgpu_ctx *ctx);
const char *pdgpu_last_error(void);
/* Device bytes currently held by the context's systems. */
int pdgpu_ctx_mem_used(pdgpu_ctx *ctx, int64_t *bytes);

/* ------------------------------------------------------------------ systems
 * A system is one WorkSpace: its atoms, topology, parameters and state.
 * Replaces the per-atom data FF_NonBonded::setup / FF_GeneralizedBorn_Still::
 * setup copy out of WorkSpace (nonbonded.cpp:1008-1036, gbff.cpp:40-87) and
 * BondOrder::reinit (workspace/bondorder.cpp:170-195).
 *   residue       Particle::ir (residue index), used for the bond-order band
 *   cov12/13/14   Particle::cov12atom/cov13atom/cov14atom as CSR (ptr[n+1],
 *                 idx), with the equilibrium distances of 1-2 and 1-3
 *                 partners (CovalentAtom::d, set by FF_Bonded::setup)
 *   gb_radius     GBtype[FFType].radius of each atom
 * The Still fixed terms (calcFixedBornRadiiTerms, gbff.cpp:307-381) and the
 * bond-order band are computed here.  *sys_id receives the handle. */
int pdgpu_system_create(pdgpu_ctx *ctx, int32_t natoms, const double *charge,
                        const double *radius, const double *epsilon,
                        const double *mass, const double *gb_radius,
                        const int32_t *residue, const int32_t *cov12_ptr,
                        const int32_t *cov12_idx, const double *cov12_d,
                        const int32_t *cov13_ptr, const int32_t *cov13_idx,
                        const double *cov13_d, const int32_t *cov14_ptr,
                        const int32_t *cov14_idx, const pdgpu_ff_params *params,
                        int32_t *sys_id);
int pdgpu_system_destroy(pdgpu_ctx *ctx, int32_t sys);
/* Change the forcefield settings (FF_NonBonded::calcCheckSum re-setup path,
 * nonbonded.cpp:1061-1067).  Topology and settings calls (set_params,
 * set_bonded, set_hydrogens, set_torsions) take single systems only. */
int pdgpu_system_set_params(pdgpu_ctx *ctx, int32_t sys, const pdgpu_ff_params *params);

/* Bonded terms as FF_Bonded::setup assembles them (ffbonded.cpp:13-470):
 * bonds (i,j | l,k), angles (i,a,j | k,theta0), torsions and impropers
 * (i,a,b,j | terms | Vn[4],n[4],gamma[4]).  Energies in J, angles in rad. */
int pdgpu_system_set_bonded(pdgpu_ctx *ctx, int32_t sys, int32_t nbond,
                            const int32_t *bond_ij, const double *bond_lk,
                            int32_t nangle, const int32_t *angle_iaj,
                            const double *angle_kt, int32_t ntors,
                            const int32_t *tors_idx, const int32_t *tors_terms,
                            const double *tors_par, int32_t nimpr,
                            const int32_t *impr_idx, const int32_t *impr_terms,
                            const double *impr_par);

/* Particle::isHydrogen() per atom (fundamentals.h:74), used by the
 * LangevinOnHydrogens=false integrator (md.cpp:1048-1218).  Default: none. */
int pdgpu_system_set_hydrogens(pdgpu_ctx *ctx, int32_t sys, const int8_t *is_h);

/* FF_SASA_LCPO (forcefields/lcpo.h, lcpo.cpp): the LCPO surface-area term,
 * epot_surf = sum over atoms of SASA_i * sigma_i.  Replaces the parameter
 * assignment of FF_SASA_LCPO::setup (lcpo.cpp:16-111): per atom, radius =
 * the LCPO type's radius + 1.4 (A), p1234 = P1..P4 ([natoms][4]), sigma =
 * the atomic solvation parameter in kcal/mol/A^2 (GlobalASP for every atom
 * on the reference's default path), use = 0 for hydrogens.  update_sasa =
 * UpdateSasa: inside the MD and minimiser loops the term is recomputed when
 * WorkSpace::Step % UpdateSasa == 0 and otherwise adds the forces of its
 * last full evaluation (lcpo.cpp:176-190); <= 0 removes the term.  Set it
 * on a single system before pdgpu_batch_create; batch members then share
 * one UpdateSasa.  With the term, pdgpu_calc_forces, pdgpu_md_run,
 * pdgpu_minimise_run and served jobs include it.  Its overlap partners come
 * from the neighbour list (the CSR rows, or the tiles of a tile search). */
int pdgpu_sasa_lcpo_set(pdgpu_ctx *ctx, int32_t sys, const double *radius,
                        const double *p1234, const double *sigma,
                        const uint8_t *use, int32_t update_sasa);
/* WorkSpace::Step for the calls outside the protocol loops
 * (pdgpu_calc_forces, pdgpu_sasa_lcpo_forces with step < 0).  Starts at 0;
 * pdgpu_md_run and pdgpu_minimise_run leave the last step they evaluated,
 * as the reference's protocols leave WorkSpace::Step. */
int pdgpu_set_step(pdgpu_ctx *ctx, int32_t sys, int32_t step);
int pdgpu_get_step(pdgpu_ctx *ctx, int32_t sys, int32_t *step);

/* ------------------------------------------------------------------ batches
 * Many independent systems of uneven size packed into one device pack
 * behind per-system offset tables, so that every kernel of an evaluation,
 * MD step or minimiser step covers all of them in one launch.  No reference
 * counterpart: the reference evaluates one WorkSpace at a time.  A batch
 * handle is used with the same calls as a system handle; per-atom arrays
 * then cover all packed atoms in member order (system s owns atoms
 * atom_offset[s] .. atom_offset[s+1]-1), and per-system outputs (energies,
 * MD history, minimiser steps) hold one record per member.  The batch takes
 * its members' topology, settings, positions, velocities and RNG keys at
 * creation and is independent of them afterwards.  Each member's results
 * equal the ones it gets alone (same pair list, same per-system reductions,
 * RNG streams keyed by the system's own key). */
int pdgpu_batch_create(pdgpu_ctx *ctx, const int32_t *sys_ids, int32_t nsys, int32_t *batch_id);
/* Member count and atom offsets (atom_offset[nsys+1]; either may be NULL). */
int pdgpu_batch_info(pdgpu_ctx *ctx, int32_t batch, int32_t *nsys, int32_t *atom_offset);
/* RNG keys of the handle's systems (seeds[nsys]); used by MD (Langevin
 * noise, initial velocities) and trial moves instead of Seed + s.  NULL
 * returns to the default keys (the MD Seed + member index). */
int pdgpu_set_seeds(pdgpu_ctx *ctx, int32_t sys, const uint64_t *seeds);

/* ------------------------------------------------------------------ trial moves
 * Backbone phi/psi rotations for Monte Carlo trial conformations
 * (MoleculeBase::setResiduePhiPsi, system/molecule.cpp:677-744, as the
 * MonteCarlo protocol's movers use it, protocols/montecarlo.cpp:16-159).
 * set_torsions lists a system's rotations from the N terminus: axis[2*k],
 * axis[2*k+1] are the bonded atoms bi, bj of the k-th bond (N-CA for phi,
 * CA-C for psi); as in MoleculeBase::rotateBond (molecule.cpp:1099-1175)
 * rotation k turns the atoms reached from bj without crossing bi about the
 * axis bj - bi.  Consecutive rotations of a chain must nest (each moves a
 * subset of what the previous one moves); a rotation that moves only atoms
 * no earlier rotation moves starts the next chain.  save_base_positions
 * keeps the current positions as the base; perturb_torsions sets the
 * positions to the base with rotation k turned by angles[k] (rad; all
 * rotations of all members in member order) or, with angles NULL, by
 * sigma * N(0,1) drawn from Philox keyed by the system's RNG key with
 * `trial` as the counter.  The result equals rotating the bonds one by one
 * from the N terminus (setResiduePhiPsi with phi+dphi, psi+dpsi). */
int pdgpu_system_set_torsions(pdgpu_ctx *ctx, int32_t sys, int32_t nrot, const int32_t *axis);
int pdgpu_save_base_positions(pdgpu_ctx *ctx, int32_t sys);
int pdgpu_perturb_torsions(pdgpu_ctx *ctx, int32_t sys, double sigma, uint64_t trial,
                           const double *angles);

/* MonteCarlo (protocols/montecarlo.h:36-125, run_core montecarlo.cpp:24-141)
 * with the phi/psi moves above as the move set and a list rebuild plus
 * Forcefield::calcForces as the evaluator, for every system of the handle
 * at once on the device.  Step 0 evaluates the starting state; step t > 0
 * perturbs the last accepted state by sigma * N(0,1) per rotation (counter
 * t, the system's RNG key).  MonteCarlo::accept (montecarlo.cpp:143-159) per
 * system: non-finite energies are rejected, lower ones accepted, otherwise
 * d = (E_old - E_new) / kB T is rejected below -50 and else accepted when a
 * uniform [0, 1) draw (Philox, keyed like the moves; the reference uses
 * rand()) is below e^d.  Temperature is a constant profile.  The handle
 * ends in FinalState (Last, LastAcc, LowestEpot) with its forces and
 * energies evaluated there.  accepted[nsys] receives the acceptances,
 * lowest[nsys] the lowest accepted epot (J); either may be NULL. */
#define PDGPU_MC_LAST 0
#define PDGPU_MC_LAST_ACC 1
#define PDGPU_MC_LOWEST_EPOT 2
typedef struct {
  int32_t Steps;
  int32_t FinalState;  /* PDGPU_MC_*; default LastAcc (montecarlo.h:53) */
  double Temperature;  /* K; default 300 */
  double Sigma;        /* rad, standard deviation of each phi/psi change; default 15 deg */
  uint64_t Seed;       /* RNG keys base + member index, unless pdgpu_set_seeds gave keys */
} pdgpu_mc_params;
void pdgpu_mc_params_default(pdgpu_mc_params *p);
int pdgpu_mc_run(pdgpu_ctx *ctx, int32_t sys, const pdgpu_mc_params *p, int32_t *accepted,
                 double *lowest);

/* State transfer (WorkSpace::cur.atom[i].p / .v / .f, snapshot.h:16-22). */
int pdgpu_set_positions(pdgpu_ctx *ctx, int32_t sys, const double *xyz);
int pdgpu_get_positions(pdgpu_ctx *ctx, int32_t sys, double *xyz);
int pdgpu_set_velocities(pdgpu_ctx *ctx, int32_t sys, const double *v);
int pdgpu_get_velocities(pdgpu_ctx *ctx, int32_t sys, double *v);
/* Forces accumulated since the last pdgpu_zero_forces, in N. */
int pdgpu_get_forces(pdgpu_ctx *ctx, int32_t sys, double *f);
/* Born radii of the last evaluation (GB_atom_param[i].bornradius). */
int pdgpu_get_born_radii(pdgpu_ctx *ctx, int32_t sys, double *born);
/* Per-atom potential energy (Particle::epot), J. */
int pdgpu_get_atom_epot(pdgpu_ctx *ctx, int32_t sys, double *epot);

/* Energy record (Hamiltonian, workspace/hamiltonian.h:23-49), J.  Index
 * order of the PDGPU_ENE_* slots below; n >= PDGPU_ENE_COUNT.  For a batch,
 * system s fills ene[s*PDGPU_ENE_COUNT ...] and n >= nsys*PDGPU_ENE_COUNT. */
#define PDGPU_ENE_EPOT 0
#define PDGPU_ENE_VDW 1
#define PDGPU_ENE_ELEC 2
#define PDGPU_ENE_POL 3
#define PDGPU_ENE_POL_CROSS 4
#define PDGPU_ENE_POL_SELF 5
#define PDGPU_ENE_BOND 6
#define PDGPU_ENE_ANGLE 7
#define PDGPU_ENE_TORSION 8
#define PDGPU_ENE_VIRIAL 9
#define PDGPU_ENE_EKIN 10
#define PDGPU_ENE_ETOT 11
#define PDGPU_ENE_GB_COMPONENT 12 /* FF_GeneralizedBorn::epot_pol of the energy path */
#define PDGPU_ENE_SURF 15         /* epot_surf (FF_SASA_LCPO) */
#define PDGPU_ENE_COUNT 16
int pdgpu_get_energies(pdgpu_ctx *ctx, int32_t sys, double *ene, int32_t n);

/* WorkSpace::zeroForces (workspace.cpp:283-292): forces, per-atom and
 * system energies to zero. */
int pdgpu_zero_forces(pdgpu_ctx *ctx, int32_t sys);

/* ------------------------------------------------------------------ kernels */
/* NeighbourList::calcNewList (neighbourlist.cpp:205-316): cell binning with
 * integer keys and a radix sort, exact FP64 distance test against
 * (max(Cutoff,VdwCutoff)+Padding)^2, bond-order encoding incl. off-diagonal
 * corrections.  Always the full ("shadow") list. */
int pdgpu_nlist_build(pdgpu_ctx *ctx, int32_t sys);
/* NeighbourListBase::getData (neighbourlist.h:47): the list in the
 * reference's packed encoding (j | bondorder<<24, j ascending per atom).
 * ptr[natoms+1]; data has room for cap entries; *count receives the total.
 * shadow=0 returns the half list (j < i) the reference builds without
 * CalcShadow. */
int pdgpu_nlist_export(pdgpu_ctx *ctx, int32_t sys, int32_t shadow, int32_t *ptr,
                       int32_t *data, int64_t cap, int64_t *count);

/* Neighbour-list build that allocates no device memory.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc, such
 * as a host framework (a simulation engine or an inference server) that
 * reserves all device memory for its own pool at start-up and forbids
 * allocation afterwards, so the caller owns every input and output buffer
 * and the library may add none of its own.  Same pair set and bond orders as
 * pdgpu_nlist_build, for one system given in device memory:
 *   x, y, z        positions (Angstrom), natoms each (SoA)
 *   list_cutoff    max(Cutoff, VdwCutoff) + Padding
 *   max_index_delta, band   BondOrder band width and band (int8,
 *                  max_index_delta * (natoms-1)), as BondOrder::getDiagData
 *   offdiag_ptr, offdiag_pairs  optional off-band partners: CSR over atoms
 *                  (natoms+1) of (partner, order) int pairs, both directions;
 *                  both NULL when there are none
 *   row_start      out: natoms+1 int64 row offsets
 *   entries        out: capacity uint32, the reference's packed entries
 *                  (j | bondorder<<24), rows in cell-scan order
 *   count          out (host): entries needed; PDGPU_ERR_ARG if > capacity
 *   stream         cudaStream_t to run on (NULL: the default stream)
 * All scratch lives in one static device array sized for 65,536 atoms
 * (about 2.9 MB, held on every GPU where the array's module is loaded, until
 * exit); larger systems are refused with PDGPU_ERR_ARG.  Calls share that
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller.  Under lazy module loading (CUDA_MODULE_LOADING=LAZY, the CUDA
 * default) the module, and with it the array, is loaded on a device by the
 * first call there or by pdgpu_ctx_create on that device, whichever comes
 * first; that is when the 2.9 MB are taken.  A caller that reserves all
 * device memory for its own pool should make one of those two calls first
 * (or run with CUDA_MODULE_LOADING=EAGER); after that the call takes no
 * device memory.  It can never run inside a stream capture: it copies small
 * host-side parameter blocks and synchronises `stream` once to read the
 * entry count. */
int pdgpu_nlist_build_noalloc(const double *x, const double *y, const double *z, int32_t natoms,
                              double list_cutoff, int32_t max_index_delta, const int8_t *band,
                              const int32_t *offdiag_ptr, const int32_t *offdiag_pairs,
                              int64_t *row_start, uint32_t *entries, int64_t capacity,
                              int64_t *count, void *stream);

/* FF_GeneralizedBorn_Still::calcForces (gbff.cpp:168-180).  FastMode (the
 * default): Born radii (:415-466), then the fused GB + LJ + Coulomb pass
 * (:1529-1736) and the Born-radius chain-rule pass (:1751-1818); adds
 * forces, sets the vdw/elec energy slots, adds the pol/pol_cross/pol_self
 * slots and their sum to EPOT.  FastMode=0: FF_NonBonded::calcForces
 * (nonbonded.cpp:1205-1229, at Dielectric = DielectricSolute, the
 * component's own switching) + calcBornForces (gbff.cpp:1172-1400: the GB
 * term without the vacuum terms, keeping its t = 0 limit q_i q_j / r
 * beyond the exp-approximation range); the LJ/Coulomb slots and the virial
 * as FF_NonBonded sets them, the GB energy added to EPOT alone (its totals
 * in the PDGPU_ENE_GB_COMPONENT slots), as the reference does. */
int pdgpu_gb_forces(pdgpu_ctx *ctx, int32_t sys);
/* FF_GeneralizedBorn_Still::calcEnergies (gbff.cpp:161-166): radii, the
 * stand-alone LJ/Coulomb pass at the solute dielectric (which, as in the
 * reference, also adds its forces), then calcBornEnergy (:520-579). */
int pdgpu_gb_energies(pdgpu_ctx *ctx, int32_t sys);
/* FF_NonBonded::calcForces (nonbonded.cpp:1205-1229, fast2 kernel :548-893):
 * VdW energy switch, electrostatics Normal / EnergySwitch / ForceSwitch /
 * distance-dependent dielectric, 1-4 scaling by bond order, virial, VdW
 * long-range correction. */
int pdgpu_nonbonded_forces(pdgpu_ctx *ctx, int32_t sys);
/* FF_Bonded::calcForces (ffbonded.cpp:809-823). */
int pdgpu_bonded_forces(pdgpu_ctx *ctx, int32_t sys);
/* FF_SASA_LCPO::calcForces (lcpo.cpp:176-190) at WorkSpace::Step = step
 * (step < 0: the handle's, pdgpu_set_step): adds its forces and adds
 * epot_cav to epot and epot_surf.  PDGPU_ERR_STATE if an atom has more than
 * 256 overlap candidates (a packing far denser than any protein's). */
int pdgpu_sasa_lcpo_forces(pdgpu_ctx *ctx, int32_t sys, int32_t step);
/* FF_SASA_LCPO::calcEnergies (lcpo.cpp:168-173, calcLCPOSasaEnergies
 * :414-566): areas and epot_surf from the energy path's overlap formula;
 * no forces. */
int pdgpu_sasa_lcpo_energies(pdgpu_ctx *ctx, int32_t sys);
/* Per-atom SASA (A^2, SASA_Atom::SASA) of the last LCPO evaluation and
 * SASAderiv of the last full one in kcal/mol/A ([natoms][3]; the reference
 * holds it in J/A and adds it / Angstrom to the force); either may be NULL. */
int pdgpu_sasa_lcpo_get(pdgpu_ctx *ctx, int32_t sys, double *sasa, double *deriv);
/* Forcefield::calcForces (forcefield.cpp:220-247) for {FF_Bonded,
 * FF_GeneralizedBorn_Still[, FF_SASA_LCPO]}: zero, bonded, GB, surface
 * term at the handle's WorkSpace::Step.  Reads nothing back. */
int pdgpu_calc_forces(pdgpu_ctx *ctx, int32_t sys);

/* ------------------------------------------------------------------ protocols */
#define PDGPU_INTEGRATOR_VERLET 0
#define PDGPU_INTEGRATOR_VELOCITY_VERLET 1
#define PDGPU_INTEGRATOR_BEEMAN 2
#define PDGPU_INTEGRATOR_LANGEVIN 3

/* MolecularDynamics public members (protocols/md.h:84-128). */
typedef struct {
  int32_t Integrator;          /* PDGPU_INTEGRATOR_*                          */
  int32_t UpdateNList;         /* rebuild the list every n steps (md.cpp:64) */
  int32_t LangevinOnHydrogens; /* md.cpp:59                                   */
  int32_t UseGraph;            /* capture UpdateNList-step blocks in a graph */
  double Timestep;             /* s                                           */
  double FricCoeff;            /* 1/s                                         */
  double TargetTemp;           /* K                                           */
  uint64_t Seed;               /* counter-based RNG key (Philox4x32-10)       */
} pdgpu_md_params;
void pdgpu_md_params_default(pdgpu_md_params *p);

/* MolecularDynamics::run_core (md.cpp:202-267): steps of {list refresh every
 * UpdateNList, Forcefield::calcForces, NaN check, integrator}.  first_step is
 * the protocol's Step of the first call; total_steps its Steps (the
 * integrators branch on Step>0 and Step<Steps-1).  Per-step epot, ekin and
 * etot (J) are written to history[3*steps*nsys] ([step][system][3]) when
 * history is not NULL.
 * Returns PDGPU_ERR_UNSTABLE on a NaN energy (assertStability,
 * protocolbase.cpp:104-110). */
int pdgpu_md_run(pdgpu_ctx *ctx, int32_t sys, const pdgpu_md_params *p,
                 int32_t first_step, int32_t steps, int32_t total_steps,
                 double *history);
/* pdgpu_md_run with the state in host memory (MolecularDynamics::run on a
 * WorkSpace whose cur state the caller owns): positions (A) and velocities
 * (m/s) in [natoms][3] are loaded first, and after the steps the positions,
 * velocities and the energy record (J, PDGPU_ENE_COUNT per system) are
 * written back.  Any pointer may be NULL to skip that transfer.  One host
 * synchronisation beyond the step loop's; page-locked buffers are copied by
 * DMA. */
int pdgpu_md_run_io(pdgpu_ctx *ctx, int32_t sys, const pdgpu_md_params *p,
                    int32_t first_step, int32_t steps, int32_t total_steps,
                    const double *x_in, const double *v_in, double *x_out,
                    double *v_out, double *ene_out);
/* Trajectory snapshots (ProtocolBase::UpdateTra with WorkSpace::outtra.append,
 * md.cpp:260 and protocolbase.cpp:229-235): with every > 0, pdgpu_md_run
 * records the positions after each step s with s > 0 and s % every == 0.
 * The integrator writes them into a device ring inside the step graph, and
 * each list period's frames are copied to a page-locked host ring of
 * `capacity` frames on the pack's second stream while the next period runs.
 * every = 0 stops recording and frees the rings. */
int pdgpu_md_set_trajectory(pdgpu_ctx *ctx, int32_t sys, int32_t every, int32_t capacity);
/* Frames recorded since the last call, oldest first: up to max_frames of
 * frames[max_frames][natoms][3] (A) with their step numbers (steps may be
 * NULL), *count of them, and *dropped (may be NULL) overwritten in the host
 * ring before they were read. */
int pdgpu_md_read_trajectory(pdgpu_ctx *ctx, int32_t sys, double *frames, int64_t *steps, int32_t max_frames,
                             int32_t *count, int32_t *dropped);
/* One integrator step with externally supplied normals (normals[6*natoms],
 * per atom in the order the reference's three nrand() pairs draw them:
 * n1x n2y n2x n1z n1y n2z), on the forces already accumulated.  For exact
 * single-step parity tests. */
int pdgpu_md_step_with_normals(pdgpu_ctx *ctx, int32_t sys, const pdgpu_md_params *p,
                               int32_t step, int32_t total_steps, const double *normals);
/* MolecularDynamics::setInitialSpeeds (md.cpp:342-363): Boltzmann draw then
 * rescale to 3/2 N kB T. */
int pdgpu_md_init_velocities(pdgpu_ctx *ctx, int32_t sys, double temperature,
                             uint64_t seed);

#define PDGPU_MIN_STEEPEST_DESCENT 0
#define PDGPU_MIN_CONJUGATE_GRADIENTS 1
/* Minimisation public members (protocols/minimise.h, minimise.cpp:34-41). */
typedef struct {
  int32_t Algorithm;
  int32_t UpdateNList;
  double StepSize;
  double SlopeCutoff;
  double Strictness;
} pdgpu_min_params;
void pdgpu_min_params_default(pdgpu_min_params *p);
/* Minimisation::runcore (minimise.cpp:99-179) with the accept / restore
 * control flow on the device; steps_taken[nsys] receives the steps each
 * system did (-1: NaN energy; a single system then returns
 * PDGPU_ERR_UNSTABLE). */
int pdgpu_minimise_run(pdgpu_ctx *ctx, int32_t sys, const pdgpu_min_params *p,
                       int32_t steps, int32_t *steps_taken);

/* ------------------------------------------------------------------ serving
 * A request loop for single-point, minimisation and MD jobs of different
 * sizes (no reference counterpart; each job runs the reference's protocol:
 * Energy::runcore energy.cpp:14-20, Minimisation::runcore minimise.cpp:
 * 99-179, MolecularDynamics::run_core md.cpp:202-267).  A worker thread owns
 * the device side of every admitted job: each job has its own stream and
 * keeps its coordinates, neighbour list, Born radii and protocol state on
 * the device until it finishes; jobs that arrive while others run are
 * admitted as soon as a stream slot is free and their memory fits under the
 * HBM budget (in arrival order, or least work -- atoms x steps -- first
 * with jobs queued for more than a second ahead of the rest), and their
 * kernels overlap with the running jobs'.  All jobs use the same pair-pass layout (and fixed
 * lanes per atom on the row layout), so a job's results are bit-identical
 * alone and in any mix.  A job's memory estimate before admission is
 * natoms * 2048 bytes + 1024 bytes per 32-atom cluster + 48 bytes per
 * possible 32 x 8 tile + 4 MiB; once its list is sized it is charged
 * max(estimate, real size).  A quarter of the slots (at least two) run on
 * the device's highest-priority streams and take single-point jobs only, so
 * those never wait behind long jobs.  With `group` set, single-point jobs
 * that are queued together, and minimisation jobs with the same settings,
 * are admitted as one batch: one pack and one launch sequence for all of
 * them, each member's results the same bits as alone.  A minimisation job's
 * chunks of 16 steps are replayed from CUDA graphs.  The server is
 * driven from one host thread (the context's). */
typedef struct pdgpu_server pdgpu_server;
typedef struct {
  int64_t hbm_budget;   /* device bytes the admitted jobs may hold together   */
  int32_t max_active;   /* jobs on the device at once (one stream each)       */
  int32_t lanes[3];     /* lanes per atom: Born, fused pair, chain (4..32)    */
  int32_t tiles;        /* 1: cluster-pair tile passes, 0: list-row passes    */
  int32_t policy;       /* admission order: 0 arrival, 1 least work first     */
  int32_t group;        /* 1: single-point jobs queued together, and
                           minimisation or MD jobs with the same settings
                           (an MD member keeps its own seed), are admitted
                           as one batch (one pack, one launch sequence;
                           tile layout only); 0: one job each             */
  int32_t batch_ms;     /* with group: a minimisation or MD job waits in the
                           queue up to this long (ms) for like jobs to
                           arrive and share its pack; 0: admitted as soon
                           as a slot is free                               */
} pdgpu_serve_params;
void pdgpu_serve_params_default(pdgpu_serve_params *p);

#define PDGPU_JOB_ENERGY 0    /* list + Forcefield::calcForces + energies          */
#define PDGPU_JOB_MINIMISE 1  /* Minimisation::runcore, `steps` steps               */
#define PDGPU_JOB_MD 2        /* MolecularDynamics::run_core, `steps` steps from
                                 velocities drawn at init_temp with md.Seed         */
typedef struct {
  int32_t kind;
  int32_t steps;
  pdgpu_md_params md;
  pdgpu_min_params min;
  double init_temp;
} pdgpu_job;

#define PDGPU_JOB_QUEUED 0
#define PDGPU_JOB_RUNNING 1
#define PDGPU_JOB_DONE 2
#define PDGPU_JOB_FAILED 3
typedef struct {
  int32_t state;        /* PDGPU_JOB_*                                          */
  int32_t status;       /* pdgpu status of a failed job                        */
  int32_t kind;
  int32_t natoms;
  int32_t steps_done;   /* MD steps / minimiser steps (-1: NaN) / 1 for energy */
  int32_t _reserved;
  double t_queue_ms;    /* submit -> admitted (-1 if not yet)                  */
  double t_run_ms;      /* admitted -> finished                                 */
  double t_total_ms;    /* submit -> finished: the job's latency               */
} pdgpu_job_info;

typedef struct {
  int64_t submitted, completed, failed;
  int32_t active, queued, peak_active;
  int32_t groups;       /* admissions that packed two or more jobs together     */
  int64_t bytes_in_use, peak_bytes;
} pdgpu_serve_stats;

int pdgpu_serve_create(pdgpu_ctx *ctx, const pdgpu_serve_params *p, pdgpu_server **out);
/* Queue a job on system `sys` (its topology and settings; a single system)
 * starting from positions xyz[3*natoms].  PDGPU_ERR_BUDGET if the job alone
 * cannot fit the budget. */
int pdgpu_serve_submit(pdgpu_server *srv, int32_t sys, const pdgpu_job *job, const double *xyz,
                       int64_t *job_id);
/* Block until the job finishes (timeout_s < 0: no limit); returns the job's
 * status. */
int pdgpu_serve_wait(pdgpu_server *srv, int64_t job_id, double timeout_s);
int pdgpu_serve_info(pdgpu_server *srv, int64_t job_id, pdgpu_job_info *info);
/* Final positions (A), forces (N), energy record (J, PDGPU_ENE_COUNT) and,
 * for MD, the per-step epot/ekin/etot history (J, 3*steps); any may be NULL. */
int pdgpu_serve_result(pdgpu_server *srv, int64_t job_id, double *xyz, double *f, double *ene,
                       double *history);
/* Forget a finished job (its host buffers return to the pool). */
int pdgpu_serve_release(pdgpu_server *srv, int64_t job_id);
int pdgpu_serve_get_stats(pdgpu_server *srv, pdgpu_serve_stats *stats);
/* Let the admitted jobs finish, fail the queued ones, stop the worker. */
int pdgpu_serve_destroy(pdgpu_server *srv);

/* ------------------------------------------------------------------ timing */
/* Device time (ms) of the last pdgpu_md_run / pdgpu_minimise_run call,
 * measured with CUDA events on the context stream. */
int pdgpu_last_run_ms(pdgpu_ctx *ctx, double *ms);

/* Instrumentation (no reference counterpart).  Pair counts of the current
 * list and positions: counts[0] = P_B, directed pairs with r <= GbsaStillCutoff
 * and bond order >= 3 (Born sum / chain rule); counts[1] = P_H, unordered
 * pairs with r <= Cutoff (fused GB + LJ + Coulomb); counts[2] = list entries;
 * counts[3] = unordered list pairs held by the cluster-pair tiles (counts[2]
 * / 2 when they agree); counts[4] = tiles (32 x 8 pair slots each). */
int pdgpu_pair_counts(pdgpu_ctx *ctx, int32_t sys, int64_t *counts);
/* Average device time (ms) of the Born-radius, fused pair and chain-rule
 * kernels over `reps` evaluations, each bracketed by CUDA events on the
 * context stream: ms[0..2]. */
int pdgpu_profile_pair_kernels(pdgpu_ctx *ctx, int32_t sys, int32_t reps, double *ms);
/* Instrumentation (no reference counterpart): device times (CUDA events on
 * the context stream, averaged over reps) of the evaluation kernel on the
 * cluster-pair tiles: ms[0..2] its Born-sum, GB + LJ + Coulomb and
 * chain-rule phases as three launches, ms[3] the three in one cooperative
 * launch (the form the protocols run).  counts (NULL, or 5 entries):
 * [0] tiles, [1] tiles the chain-rule phase visited (a pair inside the
 * Still cutoff), [2..4] tiles the Born-sum, GB + LJ + Coulomb and
 * chain-rule phases redid in their careful form (a pair at a decision
 * edge decided in FP64).  PDGPU_ERR_STATE unless the handle is on the tile
 * layout. */
int pdgpu_profile_eval(pdgpu_ctx *ctx, int32_t sys, int32_t reps, double *ms, int64_t *counts);
/* Instrumentation (no reference counterpart): the throughput of the two
 * pipes the pair kernels are bound by, measured on the context's device
 * with every SM full of warps: out[0] FP32 flop/s of fused multiply-adds
 * (2 flop each), out[1] special-function operations/s (ex2.approx), out[2]
 * the SM count.  The best of three timed launches each (a few ms). */
int pdgpu_measure_pipe_peaks(pdgpu_ctx *ctx, double *out);
/* How an evaluation on the tile layout is launched (no reference
 * counterpart): 1 = the three passes in one cooperative launch everywhere,
 * 0 = the same three phases as three launches everywhere, 2 (the default) =
 * one cooperative launch for single evaluations and minimiser / Monte Carlo
 * steps, three launches inside MD step blocks (where the next step's first
 * phase can start beside the bonded terms and the previous step's energy
 * record); -1 = only report.  Every mode gives the same bits.  *current
 * (may be NULL) receives the mode. */
int pdgpu_eval_mode(pdgpu_ctx *ctx, int32_t sys, int32_t set, int32_t *current);
/* Device times (CUDA events, averaged over reps full evaluations at step 0)
 * of the LCPO term's two launches and the work they did: out[0] overlap
 * list ms, out[1] area/derivative ms, out[2] overlap partners kept, out[3]
 * (atom, partner, partner's partner) triples of the inner loop, out[4] the
 * triples whose third atom overlaps the first (those run the whole inner
 * body).  The forces of the timed evaluations are left in the
 * accumulators. */
int pdgpu_profile_lcpo(pdgpu_ctx *ctx, int32_t sys, int32_t reps, double *out);
/* Kernels this context has launched (graph replays count their kernel
 * nodes). */
int pdgpu_launch_count(pdgpu_ctx *ctx, int64_t *count);
/* Instrumentation (no reference counterpart): step blocks of pdgpu_md_run
 * on this handle that replayed a captured graph (replays[0]) and the graphs
 * cached for it now (replays[1]).  A run cuts its steps at the list periods
 * (a rebuild every UpdateNList steps, protocolbase.cpp:113-122); every block
 * of more than one step, a partial first or last period included, replays
 * a graph when UseGraph is set. */
int pdgpu_graph_replays(pdgpu_ctx *ctx, int32_t sys, int64_t *replays);
/* Autotuner (no reference counterpart): re-time the lanes-per-atom choice
 * (4, 8, 16 or 32 lanes walk one atom's neighbour row) of the Born-radius,
 * fused pair and chain-rule kernels on the current list; lpa[0..2] receive
 * the picks.  The first force evaluation of a system tunes automatically. */
int pdgpu_autotune(pdgpu_ctx *ctx, int32_t sys, int32_t *lpa);
/* Fix the lanes per atom (lpa[0..2], each 4, 8, 16 or 32) instead of
 * tuning; NULL re-enables tuning at the next evaluation.  Results are
 * bit-identical run to run for given lanes per atom; with the same lanes a
 * system's results are bit-identical alone and in any batch. */
int pdgpu_set_lanes(pdgpu_ctx *ctx, int32_t sys, const int32_t *lpa);
/* Pair-pass layout (no reference counterpart): 0 = neighbour-list rows
 * (lanes per atom as tuned or set), 1 = cluster-pair tiles (32 x 8 atom
 * blocks of the same pair set, each unordered pair once; results do not
 * depend on lanes, row order or the batch a system sits in), -1 = let the
 * autotuner time both at the next evaluation, -2 = only report.  *current
 * (may be NULL) receives the layout in use. */
int pdgpu_pair_path(pdgpu_ctx *ctx, int32_t sys, int32_t set, int32_t *current);

#ifdef __cplusplus
}
#endif
#endif
