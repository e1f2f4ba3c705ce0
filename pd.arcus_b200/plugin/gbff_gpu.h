// FF_GeneralizedBorn_Still_GPU: PD's Still GB component with its energy and
// force evaluation on the B200 through libpdgpu's C ABI.
//
// A drop-in for Physics::FF_GeneralizedBorn_Still (forcefields/gbff.h:120-172
// of the reference): it derives from it, so every public attribute the
// reference exposes (Cutoff, InnerCutoff, VdwCutoff, VdwInnerCutoff,
// Vdw14Scaling, Elec14Scaling, DielectricSolute, DielectricSolvent,
// GbsaStillCutoff, ExpApproxThreshold, DielectricOffset, BornRadiusOffset,
// FastMode, P1..P5, EnergySwitch, ...) keeps its name and meaning, and the
// reference's protocols (MolecularDynamics, Minimisation, Energy,
// MonteCarlo) drive it through Forcefield::calcForces / calcEnergies as they
// drive the CPU component.  The ForcefieldBase contract it keeps
// (forcefield.h:93-222, gbff.cpp:160-180, 1731-1736, 1810-1816):
//   setup()         the base setup (parameter tables, Born fixed terms on the
//                   host, the list cutoff request and CalcShadow), then the
//                   system on the device: charges, LJ radii and well depths,
//                   masses, GB radii (GBtype of each atom's force-field
//                   type), residue indices and the 1-2/1-3/1-4 covalent lists
//                   with their equilibrium distances, and the settings
//   calcForces()    adds the GB + LJ + Coulomb forces (N) to
//                   wspace.cur.atom[i].f; assigns ene.epot_vdw and
//                   ene.epot_elec, adds ene.epot_pol / _pol_cross / _pol_self
//                   and the component's total to ene.epot; adds each atom's
//                   share to atom[i].epot
//   calcEnergies()  the energy-only path (Born radii, the vacuum LJ/Coulomb
//                   at DielectricSolute, calcBornEnergy): the LJ/Coulomb
//                   forces added, epot_vdw / epot_elec assigned, the total
//                   added to ene.epot
// The device keeps its own neighbour list, rebuilt at the current positions
// whenever the workspace's list has been rebuilt since the last evaluation
// (NeighbourListBase::getFullUpdateCount), so both hold the same pairs.
// A libpdgpu error becomes a ProcedureException carrying its message.
#ifndef PDGPU_GBFF_GPU_H
#define PDGPU_GBFF_GPU_H

#include "global.h"
#include "forcefields/gbff.h"

struct pdgpu_ctx;

namespace Physics {

/// the libpdgpu context of a device, shared by the components of a process
pdgpu_ctx *plugin_context(int device);

class FF_GeneralizedBorn_Still_GPU : public FF_GeneralizedBorn_Still {
 public:
  explicit FF_GeneralizedBorn_Still_GPU(WorkSpace &newwspace, int device = 0);
  FF_GeneralizedBorn_Still_GPU(const FF_GeneralizedBorn_Still_GPU &other);
  virtual ~FF_GeneralizedBorn_Still_GPU();
  virtual FF_GeneralizedBorn_Still_GPU *clone() const { return new FF_GeneralizedBorn_Still_GPU(*this); }

  /// CUDA device the component runs on
  int Device;

 protected:
  virtual void setup();
  virtual void calcForces();
  virtual void calcEnergies();

 private:
  void release();
  void upload_positions();
  void refresh_list();
  void apply_forces();
  void check(int status, const char *what) const;

  pdgpu_ctx *m_ctx;
  int m_sys;
  unsigned m_listCount;
  bool m_haveList;
  std::vector<double> m_buf;   // [3N] positions / forces in transit
  std::vector<double> m_ene;   // the device energy record (J)
  std::vector<double> m_epot;  // per-atom energies (J)
};

}  // namespace Physics

#endif
