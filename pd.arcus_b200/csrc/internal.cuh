// Internal data model of libpdgpu (B200 / sm_100a).
//
// A Pack is a set of systems resident on one device, atoms concatenated.
// Every kernel works on a Pack through PackView; per-atom arrays are SoA,
// per-system settings live in a small SysParams table indexed by sys_of[i].
// A single system is a Pack of one; batched evaluation packs many.
//
// Units inside the kernels: Angstrom, kcal/mol, kcal/mol/A, e.  Conversion
// to the reference's SI units (J, N) happens only at the C-ABI boundary.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <stdint.h>

#include <string>
#include <vector>

#include "pdgpu.h"

namespace pdgpu {

// ----------------------------------------------------------------- constants
// Values the reference computes in forcefields/forcefield.cpp:18-38 (same
// expressions, evaluated once on the host in double precision).
struct Consts {
  double kcal2J, J2kcal, Na, kB, Angstrom, econv, econv_joule, halfeconv,
      halfeconv_joule;
  double J_per_kcalmol;  // kcal2J / Na : kcal/mol -> J/molecule
  double N_per_kcalmolA; // (kcal2J/Na) / Angstrom : kcal/mol/A -> N
};
const Consts &consts();

// Fixed-point scales.  Forces: kcal/mol/A * 2^32 in int64 (range +-2.1e9
// kcal/mol/A).  Born sums: A^-1 * 2^40 in int64 (range +-8.3e6).
constexpr double kForceScale = 4294967296.0;          // 2^32
constexpr double kInvForceScale = 1.0 / 4294967296.0;
constexpr double kJScale = 16777216.0;                // 2^24: tile pass forces and energies
constexpr double kInvJScale = 1.0 / 16777216.0;
constexpr int kReduceChunk = 256;                     // items per block of the per-system reductions
constexpr int kPartSlots = 12;                        // reduction partials per (chunk, system)
constexpr int kLcpoMax = 80;                          // overlap partners kept per atom (lcpo.h Nlistmax)
constexpr int kLcpoCand = 256;                        // overlap candidates an atom may have (ranked, then cut to 80)
constexpr double kBornScale = 1099511627776.0;        // 2^40
constexpr double kInvBornScale = 1.0 / 1099511627776.0;

// Per-system settings in kernel units.  Float copies feed the FP32 pair
// math; double copies feed the exact recomputation of the two
// discontinuous predicates (Still cutoff, GB exp-approximation threshold).
struct SysParams {
  // cutoffs
  float rc2, rc, rin, inv_sw2;           // elec/GB energy switch
  float vdw_rc, vdw_rin, vdw_inv_sw2;    // VdW energy switch
  float vdw14, elec14;
  float econv_in, econv_out;             // econv / eps_solute, econv / eps_solvent
  float premul;                          // Born premultiplier, kcal/mol*A
  float exp_thresh;                      // ExpApproxThreshold
  float still2;                          // GbsaStillCutoff^2
  float P4, P5, invP5, piP5;
  // stand-alone LJ/Coulomb (FF_NonBonded)
  float econv_nb;                        // econv / Dielectric
  float ddd_alpha, dielectric;
  float fs_A, fs_B, fs_C, fs_D, fs_E, fs_cutV, fs_eshift;  // force switch
  float vdwcor_e;                        // per-atom long-range correction, kcal/mol
  int elec_mode;                         // 0 none 1 normal 2 DDD 3 energy switch 4 force switch
  int vdw_mode;                          // 0 none 2 energy switch
  int fast_mode;
  int pad_;
  // exact predicates (double)
  double still2_d, exp_thresh_d, nl_lim2_d, rc2_d;
  double halfeconv_d, born_offset_d, premul_d;
  double vdwcor_e_d;
  double P5_d, invP5_d;                  // Still P5 for the FP64 Born sums
};

enum EneSlot {
  E_EPOT = 0, E_VDW, E_ELEC, E_POL, E_POL_CROSS, E_POL_SELF, E_BOND, E_ANGLE,
  E_TORSION, E_VIRIAL, E_EKIN, E_ETOT, E_GB_COMPONENT, E_SURF = 15, E_COUNT = 16
};

// Per-atom energy terms written by the pair kernels (kcal/mol), reduced per
// system in a fixed order so every sum is bit-reproducible.
enum AtomEne { AE_VDW = 0, AE_ELEC, AE_POL, AE_POL_SELF, AE_VIR, AE_KIN, AE_SURF, AE_COUNT };

// What one energy reduction applies to the record (launch_energy).
enum EnergyMode {
  EM_PAIR_GB = 1,      // fused GB + LJ + Coulomb: vdw, elec, pol, pol_cross, pol_self
  EM_PAIR_NB = 2,      // stand-alone LJ / Coulomb: vdw, elec, virial
  EM_BORN_ENERGY = 4,  // energy-only Born term
  EM_BONDED = 8,       // bond, angle, torsion, bond virial
  EM_KINETIC = 16,     // ekin, etot
  EM_RECORD = 32,      // history row + step counter advance (step loops)
  EM_ASSIGN = 64,      // form the record from zero (its slots were not zeroed before the step)
  EM_SURF = 128,       // LCPO surface term: epot_surf
  EM_PAIR_GB_SLOW = 256  // GB with FastMode off (calcBornForces): pol + self added to epot alone;
                         // the LJ/Coulomb slots come from EM_PAIR_NB
};

// FF_SASA_LCPO (forcefields/lcpo.h, lcpo.cpp): per-atom parameters and the
// state the reference keeps between full evaluations (the overlap lists,
// each atom's SASA and SASAderiv).  A pack has the term when `update` > 0;
// batch members without it have `use` 0 on every atom.
struct LcpoView {
  int update = 0;                      // UpdateSasa: full evaluation when Step % update == 0
  int n_used = 0;                      // atoms with use = 1; the kernels run one warp per such atom
  const int *atoms = nullptr;          // [n_used] their indices, ascending (the others' state stays 0)
  const double *r = nullptr;           // [N] LCPO type radius + 1.4 (A)
  const double4 *p = nullptr;          // [N] P1..P4
  const double *sigma = nullptr;       // [N] atomic solvation parameter, kcal/mol/A^2
  const unsigned char *use = nullptr;  // [N]
  int *cnt = nullptr;                  // [N] partners kept (<= kLcpoMax)
  int *idx = nullptr;                  // [N * kLcpoMax] partners, ascending
  double *s = nullptr;                 // [N * kLcpoMax] overlap areas (A^2)
  double *sasa = nullptr;              // [N] A^2 of the last evaluation
  double *deriv = nullptr;             // [3N] SASAderiv (kcal/mol/A; x, y, z blocks) of the last full one
  double4 *xr = nullptr;               // [N] (x, y, z, r) of the heavy atoms at the last evaluation
  int *cand_n = nullptr;               // [N] candidates gathered from the tiles (0 between evaluations)
  int *cand = nullptr;                 // [N * kLcpoCand] their indices, in no order
};

// Where an evaluation takes the reference's WorkSpace::Step from: a device
// counter (the MD step, or each system's minimiser step at `stride` ints
// per system), else `imm`.
struct StepSrc {
  const int *p = nullptr;
  int stride = 0;
  int imm = 0;
};

struct BondedTerms {
  int nb = 0, na = 0, nt = 0, ni = 0;
  const int *term_off = nullptr;  // [4*(S+1)]: bond, angle, torsion, improper ranges per system
  double *e_bond = nullptr, *vir_bond = nullptr, *e_angle = nullptr, *e_dih = nullptr;
  int2 *bij = nullptr;        // bond atoms (global)
  double2 *blk = nullptr;     // (l, k kcal/mol/A^2)
  int4 *aiaj = nullptr;       // (i, a, j, -)
  double2 *akt = nullptr;     // (k kcal/mol/rad^2, theta0)
  int4 *tidx = nullptr;       // torsions then impropers (i,a,b,j)
  int *ttype = nullptr;       // [dihedrals] parameter set of each
  int *tterms = nullptr;      // [sets] Fourier terms
  double *tpar = nullptr;     // [sets * 20], 4 each: Vn kcal/mol, n, gamma, cos gamma, sin gamma
};

// Device view of a Pack.  Plain pointers, passed by value to kernels.
struct PackView {
  int n_atoms, n_sys;
  const int *atom_off;        // [S+1]
  const int *sys_of;          // [N]
  const SysParams *sp;        // [S]
  // state (FP64)
  double *x, *y, *z;          // Angstrom
  double *vx, *vy, *vz;       // m/s
  double *ox, *oy, *oz;       // saved positions (minimiser / restore)
  // pair-kernel records: one 32-byte sector per atom per gather
  float4 *pq;                 // [2N]: (x_hi, y_hi, z_hi, q), (x_lo, y_lo, z_lo, born radius)
  double4 *xyzp;              // [N]: (x, y, z, P4*V_j) for the FP64 Born sums
  float4 *chainp;             // [N]: (gb_R, V_j, gpi*deda, 0) for the chain-rule pass
  const float4 *prm;          // (lj_radius, sqrt_eps (kcal/mol)^1/2, gb_R, V_j)
  const double *gbR_d;        // gb_R (double)
  const double *pv_d;         // P4 * V_j (double)
  const double *terms123;     // Still fixed terms (A^-1 scaled like the reference)
  const double *inv_mass_si;  // 1 / kg
  const double *mass_si;      // kg
  double *born_d;             // Born radii
  long long *fx, *fy, *fz;    // fixed-point forces of the scattering terms (bonded)
  double *gx, *gy, *gz;       // pair forces (kcal/mol/A), each atom owned by one lane group
  double *fox, *foy, *foz;    // saved forces (N) for Beeman / minimiser
  double *dirx, *diry, *dirz; // CG directions / old directions
  double *odx, *ody, *odz;
  double *e_atom;             // [AE_COUNT * N]
  double *ene;                // [S * E_COUNT] J-free kcal/mol accumulators
  double *e_part;             // [S * e_chunks * kPartSlots] reduction partials
  int *e_done;                // [S] blocks of the energy reduction finished (reset by the last)
  int e_chunks;               // kReduceChunk-item chunks of the largest per-system range
  int lpa[3];                 // lanes per atom of the Born, fused-pair and chain kernels
  // backbone torsion moves (Monte Carlo trial conformations)
  const int2 *rot_axis;       // [R]: axis atoms (global) of every phi/psi rotation
  const int *rot_off;         // [S+1]: rotation range of each system
  const unsigned char *rot_start; // [R]: 1 where a nest of rotations (a chain) begins
  const int *rot_last;        // [N]: last rotation (global) that moves the atom, -1 none
  double *rot_xf;             // [R*12]: prefix-composed affine transforms
  double *bx, *by, *bz;       // base positions the trial moves start from
  // bond order
  const int *mid;             // [S]
  const long long *band_off;  // [S]
  const int8_t *band;
  const int *off_ptr;         // [N+1] off-diagonal partners per atom
  const int2 *off_data;       // (partner global index, order)
  // neighbour list (full): entries (j_global << 3) | bondorder
  long long *row_start;       // [N+1]
  int *row_cnt;               // [N]
  unsigned *nl;
  long long nl_cap;
  // cell grid
  int *cell_key;              // [N]
  int *sorted_atom;           // [N]
  int *cell_start, *cell_end; // [cell_cap]
  int cell_cap;
  double *grid;               // [S*8] origin xyz, cell size, dims(as double), cell_off
  unsigned long long *bbox;   // [6*S] ordered-integer box: min x,y,z then max x,y,z (each [S])
  // cluster-pair tiles (tiles.cu): i-clusters of 32 atoms, j-clusters of 8
  int tile_mode;              // 1: the pair passes run on the tiles, 0: on the list rows
  int n_sc;                   // i-clusters over all systems
  int max_sys_atoms;          // largest system (sizes the tile build's shared memory)
  const int *sc_atom0, *sc_sys;  // [n_sc] first atom, system
  const int *sc_jc0;          // [n_sc] first j-cluster of each i-cluster
  int n_jc;                   // j-clusters over all systems
  const int *jc_atom0;        // [n_jc] first atom of each j-cluster
  const int *jc_off;          // [S+1] first j-cluster of each system
  double *cbox;               // [6*n_jc] j-cluster boxes at the last search: lo xyz, hi xyz
  double *xs;                 // [3*N] positions at the last tile search (x block, y block, z block)
  int4 *tile_meta;           // [tile_cap] per tile: first j atom, bond-order rows index (-1 none),
                              // i-cluster's first atom, system << 8 | (i atoms - 1) << 3 | (j atoms - 1)
  unsigned *tile_rows;        // [8*tile_cap] byte l = i lane l's list bits over the 8 j atoms
  unsigned *spec_rows;        // [16*spec_cap] bytes 0..31 bond order <= 2, 32..63 == 3
  int *tile_count;            // [4] tiles, bond-order row sets, still-list length, evaluation barrier counter
  long long tile_cap, spec_cap;
  int tile_blocks[3];         // resident blocks of the three tile passes (persistent grids)
  int *still_list;            // [tile_cap] tiles with a pair inside the Still cutoff (evaluation kernel)
  int *defer_list;            // [tile_cap] tiles a warp redoes in the careful form (evaluation kernel)
  int *defer_stats;           // [3] deferred tiles per phase, counted when set (profiling only)
  int ev_blocks;              // grid of the evaluation kernel (its resident blocks)
  int ev_lean;                // every system FastMode with one switch for LJ and GB/Coulomb
  long long *bsum;            // [N] Born sums of the tile pass, fixed point 2^40
  long long *hx, *hy, *hz;    // [N] pair forces of the tile passes, fixed point 2^24 kcal/mol/A
  long long *ej;              // [4*N] LJ, Coulomb, GB energies and dE/da of the tile pass, fixed point 2^24
  int *flags;                 // [8] overflow / nan / etc.
  int *sys_flags;             // [S] SysFlag bits of the current evaluation
  // energy buffer 1 (ebuf): the evaluation kernel on the tiles and the
  // energy record of an MD step alternate between two copies of the pair
  // slots of e_atom (AE_VDW .. AE_POL_SELF) and of sys_flags, so a step's
  // record can run beside the next step's evaluation
  double *e_pair_alt;         // [4N]
  int *sys_flags_alt;         // [S]
  int ebuf;                   // 0: e_atom / sys_flags, 1: the copies (set per launch)
  BondedTerms bt;
  LcpoView lc;
};

// F_LCPO_CAND: an atom had more LCPO overlap candidates than a warp sorts
// F_BARRIER: a grid barrier of the evaluation kernel ran out of time
enum Flag { F_NL_OVERFLOW = 0, F_NAN = 1, F_CELL_CLAMP = 2, F_LCPO_CAND = 3, F_BARRIER = 4, F_COUNT = 8 };
constexpr const char *kLcpoCandMsg =
    "an atom has more than 256 LCPO overlap candidates (atoms closer than their radii + 2.8 A)";
// per system: a tile pass met a non-finite pair term (its fixed-point sums
// cannot carry it; the energy record turns it into a NaN potential energy)
enum SysFlag { SF_NONFINITE = 1 };

// ----------------------------------------------------------------- host side
struct SystemHost {
  int natoms = 0;
  pdgpu_ff_params params;
  std::vector<double> charge, radius, epsilon, mass, gbR;
  std::vector<int> residue;
  std::vector<int> c12p, c12i, c13p, c13i, c14p, c14i;
  std::vector<double> c12d, c13d;
  // derived
  int mid = 0;
  std::vector<int8_t> band;
  std::vector<int> off_i, off_j, off_o;   // unique (i<j) pairs, last order wins
  std::vector<double> vj, terms123;
  // bonded (reference units)
  std::vector<int> bij, aiaj, tidx, tterms;
  std::vector<double> blk, akt, tpar;
  int nb = 0, na = 0, nt = 0, ni = 0;
  // the dihedrals' distinct parameter sets (12 parameters and the term
  // count, 13 doubles a set, in order of first appearance) and each
  // dihedral's set, formed once when the terms are set (dihedral_sets) so
  // that building a pack maps a few sets per system instead of every term
  std::vector<int> dih_set;
  std::vector<double> dih_sets;
  // backbone torsion moves: axis atom pairs (local), nest starts and the
  // last rotation (local index, -1 none) that moves each atom
  std::vector<int> rot_axis, rot_last;
  std::vector<unsigned char> rot_start;
  std::vector<int8_t> is_h;
  // FF_SASA_LCPO: update 0 = no surface term
  int lcpo_update = 0;
  std::vector<double> lcpo_r, lcpo_p, lcpo_sigma;  // lcpo_p: [N][4]
  std::vector<unsigned char> lcpo_use;
};

// Owner of device memory for a Pack.
struct Pack {
  int device = 0;
  PackView v{};
  std::vector<int> atom_off;     // host copy
  std::vector<SysParams> sp;     // host copy
  std::vector<void *> allocs;    // stream-ordered (pooled) allocations on `st`
  cudaStream_t st = nullptr;
  int64_t bytes = 0;
  long long nl_total = -1;       // last known list size (host)
  bool have_list = false;        // a pair structure exists (list, or tiles from a search)
  bool csr_stale = false;        // the last rebuild made only the tiles (positions saved in v.xs)
  int radix_passes = 3;
  // temporary buffers for scans / sorts
  int *tmp_keys = nullptr, *tmp_vals = nullptr;
  int *sort_hist = nullptr;      // [256 * blocks]
  long long *scan_tmp = nullptr;
  int scan_tmp_len = 0;
  double *red_tmp = nullptr;     // reductions
  double *stage = nullptr;       // [3N] interleaved staging of the state transfer calls
  // bookkeeping for protocols
  unsigned char *is_h = nullptr; // Particle::isHydrogen per atom
  long long rot_total = 0;       // backbone rotations over all systems
  int nlist_counter = 0;
  bool tuned = false;            // lanes-per-atom chosen by the autotuner
  double last_run_ms = 0.0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // the bonded terms run on a second stream beside the pair passes
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // an MD step's energy record runs on the second stream beside the next
  // step's first passes; the next writer of what it reads waits on its
  // ene_done event.  On the tile layout step q of a block records from
  // energy buffer q & 1 (PackView::ebuf): the evaluation of step q + 1
  // writes the other buffer and does not wait; the evaluation of step q + 2
  // and the integrator of step q + 1 (it writes the kinetic energies the
  // record reads) do.  The row passes use buffer 0 only and wait for every
  // pending record before the fused pass.
  cudaEvent_t fork2 = nullptr, ene_done[2] = {nullptr, nullptr};
  bool ene_pending[2] = {false, false};
  int last_ebuf = 0;             // buffer of the last evaluation's per-atom energies
  bool energy_pending() const { return ene_pending[0] || ene_pending[1]; }
  // a member has FastMode off: the vacuum LJ/Coulomb come from the
  // stand-alone pass over the neighbour-list rows
  bool slow() const {
    for (const SysParams &q : sp)
      if (!q.fast_mode) return true;
    return false;
  }
  void wait_energy(cudaStream_t s, int b) {
    if (ene_pending[b]) {
      cudaStreamWaitEvent(s, ene_done[b], 0);
      ene_pending[b] = false;
    }
  }
  // evaluations may use the cooperative single-launch kernel (not for the
  // request loop's jobs, whose streams run side by side).  Inside an MD
  // step block the three-launch form is the default: its first phase starts
  // while the bonded terms and the previous step's energy record still hold
  // SMs, where a cooperative grid waits for all of its blocks to fit.
  bool coop = true;
  bool coop_md = false;
  ~Pack();
};

// Build a device Pack from host systems (atoms concatenated in order).
// With `sync` the call waits for the uploads on `st` (reporting their
// errors); without, everything stays enqueued on `st`.
// Fill h.dih_set / h.dih_sets from h.tpar and h.tterms.
void dihedral_sets(SystemHost &h);
Pack *pack_create(int device, cudaStream_t st, const std::vector<const SystemHost *> &systems,
                  std::string *err, bool sync = true);
void pack_set_params(Pack *p, int s, const pdgpu_ff_params &prm);
// allocate the cluster-pair tile store of a pack (once; enqueued on p->st)
int pack_ensure_tiles(Pack *p);
// the state transfer staging array (once; enqueued on p->st)
int pack_ensure_stage(Pack *p);
// FF_SASA_LCPO parameters of the members (again after they change)
int pack_upload_lcpo(Pack *p, const std::vector<const SystemHost *> &systems);
SysParams make_sys_params(const pdgpu_ff_params &p);

// Host setup computations (restate the reference's setup code).
int host_bondorder(SystemHost &s, std::string *err);
void host_gb_fixed_terms(SystemHost &s);

// ----------------------------------------------------------------- launchers
// All launchers enqueue on `st` and do not synchronise.
void launch_pack_positions(const PackView &v, cudaStream_t st);
// pdgpu_md_run_io's state transfer: interleaved [n][3] staging <-> the pack
void launch_state_in(const PackView &v, const double *X, const double *V, cudaStream_t st);
void launch_state_out(const PackView &v, double *X, double *V, cudaStream_t st);
void launch_aos_to_soa(const double *aos, double *X, double *Y, double *Z, int n, cudaStream_t st);
void launch_soa_to_aos(double *aos, const double *X, const double *Y, const double *Z, int n, cudaStream_t st);
void launch_zero(const PackView &v, cudaStream_t st);
// neighbour list: build phases.  count -> (host may read total) -> fill
void launch_nlist_count(Pack &p, cudaStream_t st);
void launch_nlist_fill(Pack &p, cudaStream_t st);
// GB.  zero: ZeroFlags bits; ZF_PAIRS zeroes the pair-force accumulators,
// ZF_BONDED the bonded-force accumulators, ZF_RECORD the potential-energy
// record and the system flags (together WorkSpace::zeroForces, so a step
// needs no separate zeroing launch)
enum ZeroFlags { ZF_PAIRS = 1, ZF_BONDED = 2, ZF_RECORD = 4 };
void launch_born_radii(const PackView &v, cudaStream_t st, int zero = 0);
void launch_gb_pair(const PackView &v, cudaStream_t st);
void launch_gb_chain(const PackView &v, cudaStream_t st);
// cluster-pair tile versions of the three passes (tiles.cu); the plain
// launchers above pick them when v.tile_mode is set.  tile_launch_shapes
// sets v.tile_blocks (host only: an occupancy query per pass kernel).
void tile_launch_shapes(PackView &v);
void launch_tiles_build(const PackView &v, cudaStream_t st);
// the tiles straight from the positions (no list); every system of the pack
// at most kTileSearchMaxAtoms atoms (the search tests every j-cluster box of
// a system against each of its i-clusters)
constexpr int kTileSearchMaxAtoms = 65536;
void launch_tiles_search(const PackView &v, cudaStream_t st);
void launch_tile_counts(const PackView &v, cudaStream_t st, unsigned long long *out);
void launch_born_radii_tile(const PackView &v, cudaStream_t st, int zero);
void launch_gb_pair_tile(const PackView &v, cudaStream_t st);
void launch_gb_chain_tile(const PackView &v, cudaStream_t st);
// the three tile passes as one evaluation (evaltiles.cu): Born sums, GB +
// LJ + Coulomb, chain rule, with the finish steps folded in; one
// cooperative launch when `coop` (and PDGPU_FUSED is not 0), else three
// launches of the same phases.  zero: ZeroFlags, as launch_born_radii.
cudaError_t launch_eval_tiles(const PackView &v, cudaStream_t st, int zero, bool coop);
int eval_tiles_grid(long long tile_cap);
// the three phases one launch each, timed with events on `st` (ms[0..2]),
// then the single cooperative launch (ms[3])
cudaError_t profile_eval_tiles(const PackView &v, cudaStream_t st, int reps, double *ms);
// the Born-sum phase alone (it fills the still list; instrumentation)
cudaError_t launch_born_phase_only(const PackView &v, cudaStream_t st);
cudaError_t measure_pipe_peaks(cudaStream_t st, double *out);
// one evaluation counting the tiles each phase redid in its careful form
cudaError_t count_deferred_tiles(const PackView &v, cudaStream_t st, int *stats);
// explicit lanes-per-atom variants (4, 8, 16, 32), used by the autotuner
void launch_born_radii_lpa(const PackView &v, cudaStream_t st, int zero, int lpa);
void launch_gb_pair_lpa(const PackView &v, cudaStream_t st, int lpa);
void launch_gb_chain_lpa(const PackView &v, cudaStream_t st, int lpa);
void launch_born_energy(const PackView &v, cudaStream_t st);
void launch_nonbonded(const PackView &v, cudaStream_t st, int elec_mode);
void launch_bonded_terms(const PackView &v, cudaStream_t st);
// FF_SASA_LCPO: overlap lists then areas and derivatives for the systems
// whose step is due (energy_only: the calcEnergies path, always evaluated);
// the other systems add their held derivatives to the forces.
// from_tiles: the overlap candidates come from the cluster-pair tiles of
// the last tile search (the CSR rows were not built), else from the rows.
void launch_lcpo(const PackView &v, cudaStream_t st, StepSrc step, bool energy_only, bool from_tiles);
// one of the two phases (0: overlap lists, 1: areas and derivatives)
void launch_lcpo_part(const PackView &v, cudaStream_t st, StepSrc step, bool energy_only, bool from_tiles,
                      int part);
// energies: per-atom / per-term energies into the per-system record
// (mode = EnergyMode bits); hist/step_dev only with EM_RECORD
void launch_energy(const PackView &v, cudaStream_t st, int mode, double *hist = nullptr,
                   int *step_dev = nullptr);
// integrators / minimiser
struct MDCoef {
  double dt, gamma, c0, c1, c2, varv, varr, crv, temp;
  // per-step constants of the Langevin update, formed once on the host:
  // (1 - c0/c1)/(gamma dt), c0 c2 / c1, 1/gamma, sqrt(1 - crv^2)
  double kick1, c0c2_c1, inv_gamma, sq_crv;
  int integrator, step, steps, use_normals, stochastic_h;
  unsigned long long seed;
};
void launch_md_step(const PackView &v, cudaStream_t st, const MDCoef &c, const double *normals,
                    const int *step_dev);
void launch_kinetic(const PackView &v, cudaStream_t st);
void launch_vel_init(const PackView &v, cudaStream_t st, double temp, unsigned long long seed);
void launch_vel_rescale(const PackView &v, cudaStream_t st, double temp);
void launch_check_nan(const PackView &v, cudaStream_t st);
// backbone phi/psi trial moves from the base positions (angles: optional
// explicit per-rotation angles, else sigma * N(0,1) from Philox keyed by
// the system's key with the trial number as counter)
void launch_torsion_moves(const PackView &v, cudaStream_t st, double sigma, unsigned long long trial,
                          const unsigned long long *keys, const double *angles);

// ----------------------------------------------------------------- random
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC11): 10 rounds of two 32x32->64 multiplies with the
// published multipliers and Weyl key increments.
struct U4 {
  unsigned a, b, c, d;
};
__device__ __forceinline__ U4 philox(U4 ctr, unsigned k0, unsigned k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    unsigned hi0 = __umulhi(0xD2511F53u, ctr.a), lo0 = 0xD2511F53u * ctr.a;
    unsigned hi1 = __umulhi(0xCD9E8D57u, ctr.c), lo1 = 0xCD9E8D57u * ctr.c;
    U4 n;
    n.a = hi1 ^ ctr.b ^ k0;
    n.b = lo1;
    n.c = hi0 ^ ctr.d ^ k1;
    n.d = lo0;
    ctr = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return ctr;
}
// uniform in (0, 1], like the reference's frand() (maths.cpp:256-261)
__device__ __forceinline__ double u01(unsigned x) { return ((double)x + 1.0) * (1.0 / 4294967296.0); }
// Box-Muller pair in the reference's form (maths.h:136-151)
__device__ __forceinline__ void nrand_pair(unsigned ua, unsigned ub, double &n1, double &n2) {
  double z1 = u01(ua), z2 = u01(ub);
  double l = sqrt(-2.0 * log(z1));
  double s, c;
  sincos(-2.0 * 3.14159265358979323846 * z2, &s, &c);
  n1 = l * c;
  n2 = l * s;
}

// ----------------------------------------------------------------- errors
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

}  // namespace pdgpu

// Every kernel launch goes through PDGPU_LAUNCH so the library can report
// how many of its kernels ran (graph replays add their kernel-node count).
// Launches a thread makes while it captures a graph are counted for the
// graph, not as runs.
namespace pdgpu {
std::atomic<long long> &launch_counter();
void count_launch();
void begin_capture_count();
long long end_capture_count();
}
#define PDGPU_LAUNCH(kern, grid, block, smem, stream, ...)          \
  do {                                                             \
    kern<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);      \
    ::pdgpu::count_launch();                                       \
  } while (0)

// Programmatic dependent launch for the kernels of the evaluation and step
// chain.  A kernel launched with PDGPU_LAUNCH_DEP may be scheduled while the
// kernel before it in the stream still runs; it must begin with
// PDGPU_DEP_ENTRY(), which waits until every earlier kernel of the stream
// has completed and its memory is visible (griddepcontrol.wait) before the
// kernel touches global memory, then lets the next kernel be scheduled in
// turn (griddepcontrol.launch_dependents).  The launch of kernel k+1 thus
// overlaps the run of kernel k; no kernel reads or writes anything before
// its predecessors are done.  PDGPU_PDL=0 in the environment turns the
// overlap off (plain launches).
#define PDGPU_DEP_ENTRY()                                          \
  do {                                                             \
    asm volatile("griddepcontrol.wait;" ::: "memory");             \
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); \
  } while (0)
namespace pdgpu {
bool pdl_enabled();
template <typename... KArgs, typename... Args>
inline void launch_dep(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, static_cast<Args &&>(args)...);
}
}  // namespace pdgpu
#define PDGPU_LAUNCH_DEP(kern, grid, block, smem, stream, ...)                       \
  do {                                                                              \
    ::pdgpu::launch_dep(kern, dim3(grid), dim3(block), (smem), (stream), __VA_ARGS__); \
    ::pdgpu::count_launch();                                                        \
  } while (0)

#define PDGPU_CUDA(call)                                      \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::pdgpu::cuda_fail(e_, #call); \
  } while (0)
