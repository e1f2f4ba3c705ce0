// FF_SASA_LCPO_GPU: PD's LCPO surface-area term with its evaluation on the
// B200 through libpdgpu's C ABI.
//
// A drop-in for Physics::FF_SASA_LCPO (forcefields/lcpo.h:36-125 of the
// reference): it derives from it and keeps GlobalASP and UpdateSasa.  Its
// ForcefieldBase contract (forcefield.h:93-222, lcpo.cpp:16-190):
//   setup()         the reference's setup (the 7 A list request and the
//                   parameter checks), then the per-atom LCPO parameters by
//                   the reference's rule: the first LCPOSASATYPE line of the
//                   parameter set with the atom's force-field type whose
//                   neighbour count is -1 or the atom's number of heavy
//                   covalent partners; radius = its radius + 1.4 A; P1..P4;
//                   hydrogens unused; sigma = GlobalASP (kcal/mol/A^2) on
//                   every atom.  They go to a device system of its own.
//   calcForces()    at WorkSpace::Step: the areas, their derivatives and
//                   forces on a step that is a multiple of UpdateSasa, the
//                   held forces otherwise (lcpo.cpp:176-190); adds the
//                   forces (N) and adds epot_cav to ene.epot and
//                   ene.epot_surf
//   calcEnergies()  the energy path's areas and energy, no forces
// A per-type ASP section (ASPsection_name) is not supported: setup throws.
// The device list is rebuilt whenever the workspace's is
// (NeighbourListBase::getFullUpdateCount) and also whenever an atom has
// moved far enough since the device list was built that a pair inside the
// largest overlap distance (twice the largest LCPO radius) could be missing
// from it: the device list holds pairs within 7 A plus the list padding,
// where the workspace's list, which the reference's term walks, holds pairs
// within the largest requested cutoff (the GB cutoff, in practice), so in a
// minimisation's large steps the 7 A list alone can lose overlap partners
// that the reference still sees.
#ifndef PDGPU_LCPO_GPU_H
#define PDGPU_LCPO_GPU_H

#include <vector>

#include "global.h"
#include "forcefields/lcpo.h"

struct pdgpu_ctx;

namespace Physics {

class FF_SASA_LCPO_GPU : public FF_SASA_LCPO {
 public:
  explicit FF_SASA_LCPO_GPU(WorkSpace &newwspace, int device = 0);
  FF_SASA_LCPO_GPU(const FF_SASA_LCPO_GPU &other);
  virtual ~FF_SASA_LCPO_GPU();
  virtual FF_SASA_LCPO_GPU *clone() const { return new FF_SASA_LCPO_GPU(*this); }

  /// CUDA device the component runs on
  int Device;

 protected:
  virtual void setup();
  virtual void calcForces();
  virtual void calcEnergies();

 private:
  void release();
  void upload_and_list();
  void finish();
  void check(int status, const char *what) const;

  pdgpu_ctx *m_ctx;
  int m_sys;
  unsigned m_listCount;
  bool m_haveList;
  double m_slack;             // list cutoff - the largest overlap distance (A)
  std::vector<double> m_ref;  // [3N] positions at the last device list build
  std::vector<double> m_buf;
  std::vector<double> m_ene;
};

}  // namespace Physics

#endif
