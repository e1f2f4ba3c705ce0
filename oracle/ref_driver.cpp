// Test-oracle driver: builds seeded synthetic peptide systems with the
// reference library (JonnyWideFoot/pd.arcus src/mmlib, compiled from its own
// sources by oracle/Makefile into oracle/_ref/) and dumps the reference's own
// FP64 results for them.  This file is test infrastructure: it is linked only
// against the reference library and runs only from the fixture generator
// (tests/golden/make_golden.py) and bench.py's CPU-baseline leg.
//
// Modes
//   build   build + pre-minimise a system, dump topology, parameters,
//           coordinates and every reference result the parity tests pin
//   time    rebuild a dumped system's topology, load its coordinates, and
//           time the reference MD step loop (the CPU baseline)
//   evals   rebuild a dumped system and time single-point evaluations
//           (list rebuild + calcForces), the batched scoring's CPU baseline
//   replay  rebuild a dumped system, load its coordinates and dump what
//           the reference's protocols give with it: the single-point
//           results, integrator steps, SD / CG minimisation, and a
//           MolecularDynamics::runcore run.  Built a second time with
//           PDGPU_COMPONENT (ref_driver_gpu), the same driver runs the
//           B200 GB component FF_GeneralizedBorn_Still_GPU in place of
//           the reference's: the drop-in check.
//
// The reference API calls used (all unchanged reference code):
//   FFParamSet::readLib                 forcefields/ffparam.h:571
//   NewProtein                          system/genpolymer.cpp:256-270
//   WorkSpace(System&)                  workspace/workspace.h:79
//   FF_Bonded, FF_GeneralizedBorn_Still forcefields/ffbonded.h, gbff.h:120
//   Forcefield::calcForces/calcEnergies forcefields/forcefield.cpp:212-247
//   NeighbourList::calcNewList          workspace/neighbourlist.cpp:205
//   Minimisation / MolecularDynamics    protocols/minimise.cpp, md.cpp
// Private integrator members are reached by compiling this translation unit
// with access specifiers opened, so single integrator steps can be driven
// with recorded random normals (the library objects are untouched).

#define private public
#define protected public
#include "global.h"
#include "system/system.h"
#include "system/molecule.h"
#include "system/genpolymer.h"
#include "forcefields/forcefield.h"
#include "forcefields/ffparam.h"
#include "forcefields/ffbonded.h"
#include "forcefields/gbff.h"
#include "forcefields/lcpo.h"
#include "tools/stringtool.h"
#include "workspace/workspace.h"
#include "workspace/neighbourlist.h"
#include "workspace/bondorder.h"
#include "workspace/snapshot.h"
#include "protocols/md.h"
#include "protocols/minimise.h"
#include "maths/maths.h"
#undef private
#undef protected
#ifdef PDGPU_COMPONENT
// the B200 GB and LCPO components (pd.arcus_b200/plugin) in place of the
// reference's
#include "gbff_gpu.h"
#include "lcpo_gpu.h"
typedef Physics::FF_SASA_LCPO_GPU LcpoComponent;
#else
typedef Physics::FF_SASA_LCPO LcpoComponent;
#endif

#include <sys/stat.h>
#include <sys/time.h>
#include <cmath>
#include <stdint.h>
#include <map>

using namespace Physics;
using namespace Protocol;
using Maths::dvector;

// ---------------------------------------------------------------- npy out
static std::string g_out;

static void npy_write(const std::string &name, const char *descr,
                      const std::vector<size_t> &shape, const void *data,
                      size_t elsize) {
  std::string path = g_out + "/" + name + ".npy";
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  std::string hdr = std::string("{'descr': '") + descr +
                    "', 'fortran_order': False, 'shape': (";
  size_t n = 1;
  for (size_t k = 0; k < shape.size(); k++) {
    char b[32];
    snprintf(b, sizeof b, "%zu,", shape[k]);
    hdr += b;
    if (k + 1 < shape.size()) hdr += " ";
    n *= shape[k];
  }
  hdr += "), }";
  size_t tot = 10 + hdr.size() + 1;
  size_t pad = (64 - tot % 64) % 64;
  hdr += std::string(pad, ' ');
  hdr += "\n";
  unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  fwrite(magic, 1, 8, f);
  uint16_t hl = (uint16_t)hdr.size();
  fwrite(&hl, 2, 1, f);
  fwrite(hdr.data(), 1, hdr.size(), f);
  if (n) fwrite(data, elsize, n, f);
  fclose(f);
}
static void put_d(const std::string &nm, const std::vector<double> &v,
                  std::vector<size_t> shape = std::vector<size_t>()) {
  if (shape.empty()) shape.push_back(v.size());
  npy_write(nm, "<f8", shape, v.empty() ? NULL : &v[0], 8);
}
static void put_i(const std::string &nm, const std::vector<int32_t> &v,
                  std::vector<size_t> shape = std::vector<size_t>()) {
  if (shape.empty()) shape.push_back(v.size());
  npy_write(nm, "<i4", shape, v.empty() ? NULL : &v[0], 4);
}
static void put_b(const std::string &nm, const std::vector<int8_t> &v) {
  std::vector<size_t> shape(1, v.size());
  npy_write(nm, "|i1", shape, v.empty() ? NULL : &v[0], 1);
}
static std::vector<size_t> shp(size_t a, size_t b) {
  std::vector<size_t> s;
  s.push_back(a);
  s.push_back(b);
  return s;
}

// ---------------------------------------------------------------- npy in
static std::vector<double> npy_read_d(const std::string &path, size_t *n0) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) { fprintf(stderr, "cannot read %s\n", path.c_str()); exit(2); }
  unsigned char magic[8];
  if (fread(magic, 1, 8, f) != 8) exit(2);
  uint16_t hl;
  if (fread(&hl, 2, 1, f) != 1) exit(2);
  std::string hdr(hl, ' ');
  if (fread(&hdr[0], 1, hl, f) != hl) exit(2);
  size_t p = hdr.find("'shape': (");
  size_t a = atol(hdr.c_str() + p + 10);
  size_t q = hdr.find(",", p + 10);
  size_t b = 1;
  if (hdr[q + 1] == ' ' && hdr[q + 2] != ')') b = atol(hdr.c_str() + q + 2);
  std::vector<double> v(a * b);
  if (fread(&v[0], 8, v.size(), f) != v.size()) exit(2);
  fclose(f);
  if (n0) *n0 = a;
  return v;
}

// ---------------------------------------------------------------- seeded RNG
// splitmix64 (Steele, Lea, Flood 2014); only used to draw sequences and
// placements, never inside the reference's own arithmetic.
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
  }
};

static std::string random_sequence(uint64_t seed, int nres) {
  static const char *aa = "ACDEFGHIKLMNPQRSTVWY";
  Rng r(seed);
  std::string s;
  for (int i = 0; i < nres; i++) s += aa[r.next() % 20];
  return s;
}
static std::string pd_seq(const std::string &s) {
  // "*X-(...)-Z*": N-terminal residue, body, C-terminal residue
  // (the form used by the reference's own examples).
  return "*" + s.substr(0, 1) + "-(" + s.substr(1, s.size() - 2) + ")-" +
         s.substr(s.size() - 1) + "*";
}

// ---------------------------------------------------------------- settings
struct Settings {
  double cutoff, inner;
  double vdwcut, vdwinner;
  std::string param;
  bool fastmode;
  Settings()
      : cutoff(12), inner(9), vdwcut(12), vdwinner(9),
        param("amber99aa.ff"), fastmode(true) {}
};

struct Built {
  FFParamSet *ffps;
  System *sys;
  WorkSpace *ws;
  Forcefield *ff;
  FF_Bonded *bonded;
  FF_GeneralizedBorn_Still *gb;
};

static void configure_gb(FF_GeneralizedBorn_Still &gb, const Settings &st) {
  gb.Cutoff = st.cutoff;
  gb.InnerCutoff = st.inner;
  gb.VdwCutoff = st.vdwcut;
  gb.VdwInnerCutoff = st.vdwinner;
  gb.FastMode = st.fastmode;
}

static Built make_ws(FFParamSet *ffps, const std::vector<std::string> &seqs,
                     const Settings &st, bool with_bonded = true) {
  Built b;
  b.ffps = ffps;
  b.sys = new System(*ffps);
  for (size_t k = 0; k < seqs.size(); k++)
    b.sys->add(NewProtein(*ffps, pd_seq(seqs[k])));
  b.ws = new WorkSpace(*b.sys);
  b.ff = new Forcefield(*b.ws);
  b.bonded = new FF_Bonded(*b.ws);
#ifdef PDGPU_COMPONENT
  b.gb = new FF_GeneralizedBorn_Still_GPU(*b.ws);
#else
  b.gb = new FF_GeneralizedBorn_Still(*b.ws);
#endif
  configure_gb(*b.gb, st);
  if (with_bonded) b.ff->add(*b.bonded);
  b.ff->add(*b.gb);
  return b;
}

static std::vector<double> get_pos(WorkSpace &ws) {
  std::vector<double> p(ws.nAtoms() * 3);
  for (size_t i = 0; i < ws.nAtoms(); i++) {
    p[3 * i] = ws.cur.atom[i].p.x;
    p[3 * i + 1] = ws.cur.atom[i].p.y;
    p[3 * i + 2] = ws.cur.atom[i].p.z;
  }
  return p;
}
static void set_pos(WorkSpace &ws, const std::vector<double> &p) {
  for (size_t i = 0; i < ws.nAtoms(); i++)
    ws.cur.atom[i].p.setTo(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
static std::vector<double> get_f(WorkSpace &ws) {
  std::vector<double> p(ws.nAtoms() * 3);
  for (size_t i = 0; i < ws.nAtoms(); i++) {
    p[3 * i] = ws.cur.atom[i].f.x;
    p[3 * i + 1] = ws.cur.atom[i].f.y;
    p[3 * i + 2] = ws.cur.atom[i].f.z;
  }
  return p;
}
static std::vector<double> get_v(WorkSpace &ws) {
  std::vector<double> p(ws.nAtoms() * 3);
  for (size_t i = 0; i < ws.nAtoms(); i++) {
    p[3 * i] = ws.cur.atom[i].v.x;
    p[3 * i + 1] = ws.cur.atom[i].v.y;
    p[3 * i + 2] = ws.cur.atom[i].v.z;
  }
  return p;
}
static void set_v(WorkSpace &ws, const std::vector<double> &p) {
  for (size_t i = 0; i < ws.nAtoms(); i++)
    ws.cur.atom[i].v.setTo(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
static std::vector<double> ene_vec(const Hamiltonian &e) {
  double a[] = {e.epot,         e.epot_vdw,  e.epot_elec, e.epot_pol,
                e.epot_pol_cross, e.epot_pol_self, e.epot_bond,
                e.epot_angle,   e.epot_torsion, e.InternalVirial};
  return std::vector<double>(a, a + 10);
}

// SD pre-minimisation used to relax the clashing extended builds.
static void preminimise(Built &b, int steps) {
  b.ff->ensuresetup(*b.ws);
  Minimisation m(*b.ff);
  m.Algorithm = Minimisation::SteepestDescent;
  m.Steps = steps;
  m.UpdateScr = 0;
  m.OutputLevel = Verbosity::Silent;
  m.runcore();
}

// Rotate a chain so its principal axis is along z, centred on (cx, cy, 0).
static void place_chain(std::vector<double> &p, double cx, double cy) {
  size_t n = p.size() / 3;
  double c[3] = {0, 0, 0};
  for (size_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) c[k] += p[3 * i + k] / n;
  double C[3][3] = {{0}};
  for (size_t i = 0; i < n; i++)
    for (int a = 0; a < 3; a++)
      for (int bb = 0; bb < 3; bb++)
        C[a][bb] += (p[3 * i + a] - c[a]) * (p[3 * i + bb] - c[bb]);
  double v[3] = {0.3, 0.5, 0.8};
  for (int it = 0; it < 200; it++) {
    double w[3];
    for (int a = 0; a < 3; a++)
      w[a] = C[a][0] * v[0] + C[a][1] * v[1] + C[a][2] * v[2];
    double nn = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    for (int a = 0; a < 3; a++) v[a] = w[a] / nn;
  }
  // rotation taking v onto z (Rodrigues)
  double z[3] = {0, 0, 1};
  double ax[3] = {v[1] * z[2] - v[2] * z[1], v[2] * z[0] - v[0] * z[2],
                  v[0] * z[1] - v[1] * z[0]};
  double s = sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
  double co = v[2];
  double R[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (s > 1e-12) {
    for (int a = 0; a < 3; a++) ax[a] /= s;
    double K[3][3] = {{0, -ax[2], ax[1]}, {ax[2], 0, -ax[0]}, {-ax[1], ax[0], 0}};
    for (int a = 0; a < 3; a++)
      for (int bb = 0; bb < 3; bb++) {
        double kk = 0;
        for (int m = 0; m < 3; m++) kk += K[a][m] * K[m][bb];
        R[a][bb] += s * K[a][bb] + (1 - co) * kk;
      }
  }
  for (size_t i = 0; i < n; i++) {
    double d[3] = {p[3 * i] - c[0], p[3 * i + 1] - c[1], p[3 * i + 2] - c[2]};
    double r[3];
    for (int a = 0; a < 3; a++) r[a] = R[a][0] * d[0] + R[a][1] * d[1] + R[a][2] * d[2];
    p[3 * i] = r[0] + cx;
    p[3 * i + 1] = r[1] + cy;
    p[3 * i + 2] = r[2];
  }
}

// ---------------------------------------------------------------- dumps
static void dump_topology(Built &b, const Settings &st) {
  WorkSpace &ws = *b.ws;
  size_t n = ws.nAtoms();
  std::vector<double> q(n), rad(n), eps(n), mass(n), gbr(n);
  std::vector<int32_t> ir(n), ffty(n);
  std::vector<int8_t> ish(n);
  std::vector<int32_t> c12p(1, 0), c13p(1, 0), c14p(1, 0), c12i, c13i, c14i;
  std::vector<double> c12d, c13d;
  for (size_t i = 0; i < n; i++) {
    const Particle &a = ws.atom[i];
    q[i] = a.charge;
    rad[i] = a.radius;
    eps[i] = a.epsilon;
    mass[i] = a.mass;
    gbr[i] = b.gb->GBtype[a.FFType].radius;
    ir[i] = a.ir;
    ffty[i] = a.FFType;
    ish[i] = a.isHydrogen() ? 1 : 0;
    for (size_t k = 0; k < a.cov12atom.size(); k++) {
      c12i.push_back(a.cov12atom[k].i);
      c12d.push_back(a.cov12atom[k].d);
    }
    for (size_t k = 0; k < a.cov13atom.size(); k++) {
      c13i.push_back(a.cov13atom[k].i);
      c13d.push_back(a.cov13atom[k].d);
    }
    for (size_t k = 0; k < a.cov14atom.size(); k++)
      c14i.push_back(a.cov14atom[k].i);
    c12p.push_back(c12i.size());
    c13p.push_back(c13i.size());
    c14p.push_back(c14i.size());
  }
  put_d("charge", q);
  put_d("radius", rad);
  put_d("epsilon", eps);
  put_d("mass", mass);
  put_d("gb_radius", gbr);
  put_i("ir", ir);
  put_i("fftype", ffty);
  put_b("is_h", ish);
  put_i("cov12_ptr", c12p);
  put_i("cov12_idx", c12i);
  put_d("cov12_d", c12d);
  put_i("cov13_ptr", c13p);
  put_i("cov13_idx", c13i);
  put_d("cov13_d", c13d);
  put_i("cov14_ptr", c14p);
  put_i("cov14_idx", c14i);
  // backbone N, CA, C of every residue (-1 where absent), for phi/psi moves
  {
    int nres = 0;
    for (size_t i = 0; i < n; i++) nres = std::max(nres, ws.atom[i].ir + 1);
    std::vector<int32_t> bb(3 * (size_t)nres, -1);
    for (size_t i = 0; i < n; i++) {
      const std::string &nm = ws.atom[i].pdbname;
      int k = nm == "N" ? 0 : (nm == "CA" ? 1 : (nm == "C" ? 2 : -1));
      if (k >= 0 && bb[3 * ws.atom[i].ir + k] < 0) bb[3 * ws.atom[i].ir + k] = (int32_t)i;
    }
    put_i("backbone_ncac", bb, shp(nres, 3));
  }

  // bond-order band matrix + off-diagonal list, as the reference built them
  const BondOrder &bo = ws.bondorder();
  std::vector<int32_t> mid(1, bo.getMaxIndexDelta());
  put_i("bo_mid", mid);
  const std::vector<char> &band = bo.getDiagData();
  std::vector<int8_t> bandv(band.begin(), band.end());
  put_b("bo_band", bandv);
  std::vector<int32_t> offd;
  const std::vector<LongBondOrder> &sp = bo.getOffDiagData();
  for (size_t p = 0; p < sp.size(); p++)
    for (size_t r = 0; r < sp[p].partner.size(); r++) {
      offd.push_back(sp[p].i);
      offd.push_back(sp[p].partner[r].j);
      offd.push_back(sp[p].partner[r].order);
    }
  put_i("bo_offdiag", offd, shp(offd.size() / 3, 3));

  // bonded terms as FF_Bonded::setup assembled them
  FF_Bonded &fb = *b.bonded;
  std::vector<int32_t> bij;
  std::vector<double> blk;
  for (size_t k = 0; k < fb.bond.size(); k++) {
    bij.push_back(fb.bond[k].i);
    bij.push_back(fb.bond[k].j);
    blk.push_back(fb.bond[k].l);
    blk.push_back(fb.bond[k].k);
  }
  put_i("bond_ij", bij, shp(bij.size() / 2, 2));
  put_d("bond_lk", blk, shp(blk.size() / 2, 2));
  std::vector<int32_t> aij;
  std::vector<double> akt;
  for (size_t k = 0; k < fb.angle.size(); k++) {
    aij.push_back(fb.angle[k].i);
    aij.push_back(fb.angle[k].a);
    aij.push_back(fb.angle[k].j);
    akt.push_back(fb.angle[k].k);
    akt.push_back(fb.angle[k].theta0);
  }
  put_i("angle_iaj", aij, shp(aij.size() / 3, 3));
  put_d("angle_kt", akt, shp(akt.size() / 2, 2));
  for (int which = 0; which < 2; which++) {
    std::vector<Torsion> &T = which == 0 ? fb.torsion : fb.improper;
    std::vector<int32_t> ti, tt;
    std::vector<double> tp;
    for (size_t k = 0; k < T.size(); k++) {
      ti.push_back(T[k].i);
      ti.push_back(T[k].a);
      ti.push_back(T[k].b);
      ti.push_back(T[k].j);
      tt.push_back(T[k].terms);
      for (int m = 0; m < 4; m++) tp.push_back(m < T[k].terms ? T[k].Vn[m] : 0.0);
      for (int m = 0; m < 4; m++) tp.push_back(m < T[k].terms ? T[k].n[m] : 0.0);
      for (int m = 0; m < 4; m++) tp.push_back(m < T[k].terms ? T[k].gamma[m] : 0.0);
    }
    std::string pre = which == 0 ? "tors" : "impr";
    put_i(pre + "_idx", ti, shp(ti.size() / 4, 4));
    put_i(pre + "_terms", tt);
    put_d(pre + "_par", tp, shp(tp.size() / 12, 12));
  }

  // GB setup-time terms
  std::vector<double> vj(n), t123(n);
  for (size_t i = 0; i < n; i++) {
    vj[i] = b.gb->GB_atom_param_still[i].Vj;
    t123[i] = b.gb->GB_atom_param_still[i].terms123;
  }
  put_d("gb_vj", vj);
  put_d("gb_terms123", t123);

  double pp[] = {b.gb->P1, b.gb->P2, b.gb->P3, b.gb->P4, b.gb->P5,
                 b.gb->Vdw14Scaling, b.gb->Elec14Scaling};
  put_d("ff_params", std::vector<double>(pp, pp + 7));
  (void)st;
}

static void dump_nlist(Built &b, const std::string &nm) {
  WorkSpace &ws = *b.ws;
  const NeighbourData *fn = ws.nlist().getData();
  std::vector<int32_t> ptr(1, 0), data;
  for (size_t i = 0; i < ws.nAtoms(); i++) {
    for (int k = 0; k < fn[i].n; k++) data.push_back(fn[i].i[k]);
    ptr.push_back(data.size());
  }
  put_i(nm + "_ptr", ptr);
  put_i(nm + "_data", data);
}

static std::vector<double> born(Built &b) {
  std::vector<double> v(b.ws->nAtoms());
  for (size_t i = 0; i < v.size(); i++) v[i] = b.gb->GB_atom_param[i].bornradius;
  return v;
}

// All single-point reference results for the current coordinates.
static void dump_single_point(Built &b, const std::string &pre) {
  WorkSpace &ws = *b.ws;
  ws.nlist().calcNewList();
  dump_nlist(b, pre + "nl");
  // full forcefield (bonded + GB) forces path
  b.ff->calcForces();
  put_d(pre + "f_total", get_f(ws), shp(ws.nAtoms(), 3));
  put_d(pre + "ene_total", ene_vec(ws.ene));
  put_d(pre + "born", born(b));
  std::vector<double> ae(ws.nAtoms());
  for (size_t i = 0; i < ae.size(); i++) ae[i] = ws.atom[i].epot;
  put_d(pre + "atom_epot", ae);
  // GB component alone
  ws.zeroForces();
  b.gb->calcForces();
  put_d(pre + "f_gb", get_f(ws), shp(ws.nAtoms(), 3));
  put_d(pre + "ene_gb", ene_vec(ws.ene));
  // bonded component alone
  ws.zeroForces();
  b.bonded->calcForces();
  put_d(pre + "f_bonded", get_f(ws), shp(ws.nAtoms(), 3));
  put_d(pre + "ene_bonded", ene_vec(ws.ene));
  // energy-only path of the GB component (radii + fast2 LJ/Coulomb + Born energy)
  ws.zeroForces();
  b.gb->calcEnergies();
  put_d(pre + "f_energypath", get_f(ws), shp(ws.nAtoms(), 3));
  std::vector<double> e = ene_vec(ws.ene);
  e.push_back(b.gb->epot_pol);
  e.push_back(b.gb->epot_pol_cross);
  e.push_back(b.gb->epot_pol_self);
  put_d(pre + "ene_energypath", e);
}

// Monte Carlo trial conformations: from the base coordinates, every
// residue's phi and psi turned by its own normal deviate (sigma, radians)
// through MoleculeBase::setResiduePhiPsi (molecule.cpp:702-711), residues
// in order; then the single-point forces of each trial.  The deviates come
// from splitmix64 + Box-Muller and are stored with the results.
static uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double normal01(uint64_t &x) {
  double u1 = ((splitmix64(x) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
  double u2 = (splitmix64(x) >> 11) * (1.0 / 9007199254740992.0);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
}
static void dump_trials(Built &b, const std::vector<double> &base, int ntrials, double sigma, uint64_t seed) {
  WorkSpace &ws = *b.ws;
  size_t n = ws.nAtoms();
  int nres = ws.nResidues();
  std::vector<double> ang, pos, f, ene;
  uint64_t state = seed * 0x2545F4914F6CDD1DULL + 12345;
  for (int t = 0; t < ntrials; t++) {
    set_pos(ws, base);
    for (int ir = 0; ir < nres; ir++) {
      double dphi = sigma * normal01(state), dpsi = sigma * normal01(state);
      double fphi, fpsi;
      ws.calcResiduePhiPsi(ir, fphi, fpsi);
      ws.setResiduePhiPsi(ir, fphi + dphi, fpsi + dpsi);
      ang.push_back(dphi);
      ang.push_back(dpsi);
    }
    std::vector<double> p = get_pos(ws);
    pos.insert(pos.end(), p.begin(), p.end());
    ws.nlist().calcNewList();
    b.ff->calcForces();
    std::vector<double> ft = get_f(ws), et = ene_vec(ws.ene);
    f.insert(f.end(), ft.begin(), ft.end());
    ene.insert(ene.end(), et.begin(), et.end());
  }
  std::vector<size_t> s3(3);
  s3[0] = ntrials;
  s3[1] = n;
  s3[2] = 3;
  put_d("trial_angles", ang, shp(ntrials, 2 * nres));
  put_d("trial_pos", pos, s3);
  put_d("trial_f", f, s3);
  put_d("trial_ene", ene, shp(ntrials, 10));
  set_pos(ws, base);
}

// One integrator step with the normals the reference's nrand() will draw,
// recorded by replaying the same srand() seed (rand() is only called by the
// Langevin step inside applyForces).
static void dump_md_steps(Built &b, int integrator, int nsteps, double fric,
                          const std::string &pre) {
  WorkSpace &ws = *b.ws;
  size_t n = ws.nAtoms();
  MolecularDynamics md(*b.ff);
  md.Integrator = (MolecularDynamics::IntegratorType)integrator;
  md.Timestep = 1e-15;
  md.FricCoeff = fric;
  md.Steps = nsteps;
  md.UpdateNList = 10;
  md.OutputLevel = Verbosity::Silent;
  // initial velocities: Boltzmann draw by the reference itself
  srand(12345);
  md.setInitialSpeeds(300.0);
  ws.old = ws.cur;  // Beeman/Verlet read old.f / old.p
  for (size_t i = 0; i < n; i++) ws.old.atom[i].f.setTo(0, 0, 0);
  put_d(pre + "v0", get_v(ws), shp(n, 3));
  put_d(pre + "x0", get_pos(ws), shp(n, 3));
  std::vector<double> xs, vs, fs, norms, ekin, epot;
  for (int s = 0; s < nsteps; s++) {
    md.Step = s;
    ws.Step = s;
    md.refreshNeighborList();
    b.ff->calcForces();
    std::vector<double> fnow = get_f(ws);
    fs.insert(fs.end(), fnow.begin(), fnow.end());
    epot.push_back(ws.ene.epot);
    // record the normals this step will draw
    srand(777 + s);
    for (size_t i = 0; i < n; i++) {
      double a1, a2, a3, a4, a5, a6;
      Maths::nrand(a1, a2, (double)1);
      Maths::nrand(a3, a4, (double)1);
      Maths::nrand(a5, a6, (double)1);
      double rec[6] = {a1, a2, a3, a4, a5, a6};
      norms.insert(norms.end(), rec, rec + 6);
    }
    srand(777 + s);
    md.applyForces();
    ekin.push_back(ws.ene.ekin);
    std::vector<double> xnow = get_pos(ws), vnow = get_v(ws);
    xs.insert(xs.end(), xnow.begin(), xnow.end());
    vs.insert(vs.end(), vnow.begin(), vnow.end());
  }
  std::vector<size_t> s3;
  s3.push_back(nsteps);
  s3.push_back(n);
  s3.push_back(3);
  put_d(pre + "x", xs, s3);
  put_d(pre + "v", vs, s3);
  put_d(pre + "f", fs, s3);
  std::vector<size_t> s6;
  s6.push_back(nsteps);
  s6.push_back(n);
  s6.push_back(6);
  put_d(pre + "normals", norms, s6);
  put_d(pre + "ekin", ekin);
  put_d(pre + "epot", epot);
}

static void dump_minimise(Built &b, int algo, int nsteps, const std::string &pre) {
  WorkSpace &ws = *b.ws;
  Minimisation m(*b.ff);
  m.Algorithm = (Minimisation::MinType)algo;
  m.Steps = nsteps;
  m.UpdateScr = 0;
  m.OutputLevel = Verbosity::Silent;
  put_d(pre + "x0", get_pos(ws), shp(ws.nAtoms(), 3));
  int taken = m.runcore();
  put_d(pre + "x", get_pos(ws), shp(ws.nAtoms(), 3));
  std::vector<double> r;
  r.push_back(taken);
  r.push_back(ws.ene.epot);
  r.push_back(m.m_StepMultiplier);
  put_d(pre + "result", r);
}

// FF_SASA_LCPO (forcefields/lcpo.cpp) on the built system.  The per-atom
// parameters its setup() derives (lcpo.cpp:16-91) are formed here from the
// parameter file's LCPOSASAPARAMETERS section with the same rule: the first
// LCPOSASATYPE line with the atom's force-field type whose neighbour count
// is -1 or the atom's number of non-hydrogen covalent partners; radius +
// 1.4; hydrogens unused.  They are not read from the component (its arrays
// are private); the oracle's energies and forces from them, compared with
// the component's own, are what checks them.  Dumped: the parameters, the
// component's forces and energies alone (calcForces at Step 0, calcEnergies),
// then the whole forcefield with it (single point, velocity-Verlet steps,
// steepest-descent steps) at UpdateSasa = update.
struct LcpoType {
  int attype, nb;
  double r, p[4];
};
static void dump_lcpo(Built &b, const std::vector<double> &allpos, double asp, int update, int steps,
                      bool dense) {
  WorkSpace &ws = *b.ws;
  size_t n = ws.nAtoms();
  Section sec;
  if (b.ffps->getSection("LCPOSASAPARAMETERS", sec) != 0) {
    fprintf(stderr, "no LCPOSASAPARAMETERS section\n");
    exit(2);
  }
  std::vector<LcpoType> types;
  for (size_t l = 0; l < sec.sectionline.size(); l++) {
    std::string line = sec.sectionline[l];
    removecomments(line, "#\12\15");
    std::vector<std::string> tok = chopstr(line, " \12\15\t");
    if (tok.size() < 8 || !cmpstring(tok[0], "LCPOSASATYPE")) continue;
    LcpoType t;
    t.attype = b.ffps->findAtomType(tok[1]);
    t.nb = atoi(tok[2].c_str());
    t.r = strtod(tok[3].c_str(), NULL);
    for (int k = 0; k < 4; k++) t.p[k] = strtod(tok[4 + k].c_str(), NULL);
    types.push_back(t);
  }
  std::vector<double> rad(n), p4(4 * n);
  std::vector<int8_t> use(n);
  for (size_t i = 0; i < n; i++) {
    const Particle &a = ws.atom[i];
    int heavy = 0;
    for (size_t k = 0; k < a.cov12atom.size(); k++)
      if (ws.atom[a.cov12atom[k].i].Z != 1) heavy++;
    size_t t = 0;
    for (; t < types.size(); t++)
      if (types[t].attype == a.FFType && (types[t].nb < 0 || types[t].nb == heavy)) break;
    if (t == types.size()) {
      fprintf(stderr, "no LCPO type for atom %zu\n", i);
      exit(2);
    }
    rad[i] = types[t].r + 1.4;
    for (int k = 0; k < 4; k++) p4[4 * i + k] = types[t].p[k];
    use[i] = a.Z == 1 ? 0 : 1;
  }
  put_d("lcpo_radius", rad);
  put_d("lcpo_p", p4, shp(n, 4));
  put_b("lcpo_use", use);
  std::vector<double> cfg;
  cfg.push_back(asp);
  cfg.push_back(update);
  put_d("lcpo_cfg", cfg);

  FF_SASA_LCPO *sasa = new FF_SASA_LCPO(ws);
  sasa->GlobalASP = asp;
  sasa->UpdateSasa = update;
  Forcefield *alone = new Forcefield(ws);
  alone->add(*sasa);
  set_pos(ws, allpos);
  alone->ensuresetup(ws);
  ws.Step = 0;
  ws.nlist().calcNewList();
  alone->calcForces();
  std::vector<double> e = ene_vec(ws.ene);
  e.push_back(ws.ene.epot_surf);
  put_d("lcpo_f", get_f(ws), shp(n, 3));
  put_d("lcpo_ene", e);
  ws.zeroForces();
  alone->calcEnergies();
  e = ene_vec(ws.ene);
  e.push_back(ws.ene.epot_surf);
  put_d("lcpo_ene_energypath", e);

  // an artificially dense packing (the coordinates shrunk to 0.35 about
  // their centroid): atoms with more than 80 overlapping partners, whose
  // overlap lists the reference truncates (lcpo.cpp:465-482)
  if (dense) {
    std::vector<double> dp(allpos);
    double c[3] = {0, 0, 0};
    for (size_t i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) c[k] += dp[3 * i + k];
    for (int k = 0; k < 3; k++) c[k] /= (double)n;
    for (size_t i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) dp[3 * i + k] = c[k] + 0.35 * (dp[3 * i + k] - c[k]);
    set_pos(ws, dp);
    ws.Step = 0;
    ws.nlist().calcNewList();
    dump_nlist(b, "lcpo_dense_nl");
    alone->calcForces();
    e = ene_vec(ws.ene);
    e.push_back(ws.ene.epot_surf);
    put_d("lcpo_dense_pos", dp, shp(n, 3));
    put_d("lcpo_dense_f", get_f(ws), shp(n, 3));
    put_d("lcpo_dense_ene", e);
    ws.zeroForces();
    alone->calcEnergies();
    e = ene_vec(ws.ene);
    e.push_back(ws.ene.epot_surf);
    put_d("lcpo_dense_ene_energypath", e);
  }

  b.ff->add(*sasa);
  b.ff->ensuresetup(ws);
  set_pos(ws, allpos);
  ws.Step = 0;
  ws.nlist().calcNewList();
  b.ff->calcForces();
  e = ene_vec(ws.ene);
  e.push_back(ws.ene.epot_surf);
  put_d("lcpo_f_total", get_f(ws), shp(n, 3));
  put_d("lcpo_ene_total", e);
  if (steps > 0) {
    set_pos(ws, allpos);
    dump_md_steps(b, MolecularDynamics::VelocityVerlet, steps, 1e12, "lcpo_mdvv_");
    set_pos(ws, allpos);
    ws.Step = 0;
    dump_minimise(b, Minimisation::SteepestDescent, steps, "lcpo_minsd_");
  }
  set_pos(ws, allpos);
}

// FF_NonBonded alone in each of its calcForces modes (nonbonded.cpp:
// 1205-1229 selects ForceSwitch over EnergySwitch over plain Coulomb; the
// DDDielectric flag is not consulted there), at the GB component's cutoffs,
// and the GB component with FastMode off (calcForces = FF_NonBonded::
// calcForces + calcBornForces, gbff.cpp:168-180, 1172-1400).
static void dump_nb_case(Built &b, const std::string &pre, bool fs, bool es, bool ddd, double diel,
                         bool vdwcor) {
  WorkSpace &ws = *b.ws;
  FF_NonBonded *nb = new FF_NonBonded(ws);
  nb->Cutoff = b.gb->Cutoff;
  nb->InnerCutoff = b.gb->InnerCutoff;
  nb->VdwCutoff = b.gb->VdwCutoff;
  nb->VdwInnerCutoff = b.gb->VdwInnerCutoff;
  nb->ForceSwitch = fs;
  nb->EnergySwitch = es;
  nb->DDDielectric = ddd;
  nb->Dielectric = diel;
  if (vdwcor) {
    nb->VdwCor = true;
    nb->VdwCorDensity = 0.0334;  // particles / A^3
    nb->VdwCorEpsilon = 0.152;   // kcal/mol
    nb->VdwCorRadius = 1.77;     // A
    nb->VdwCorCutoff = nb->VdwCutoff;
  }
  Forcefield ff(ws);
  ff.add(*nb);
  ff.ensuresetup(ws);
  ws.nlist().calcNewList();
  ff.calcForces();
  put_d(pre + "f", get_f(ws), shp(ws.nAtoms(), 3));
  put_d(pre + "ene", ene_vec(ws.ene));
  std::vector<double> cfg;
  cfg.push_back(nb->Cutoff);
  cfg.push_back(nb->InnerCutoff);
  cfg.push_back(fs);
  cfg.push_back(es);
  cfg.push_back(ddd);
  cfg.push_back(diel);
  cfg.push_back(vdwcor);
  cfg.push_back(nb->VdwCorDensity);
  cfg.push_back(nb->VdwCorEpsilon);
  cfg.push_back(nb->VdwCorRadius);
  cfg.push_back(nb->VdwCorCutoff);
  cfg.push_back(nb->Vdw14Scaling);
  cfg.push_back(nb->Elec14Scaling);
  put_d(pre + "cfg", cfg);
}
static void dump_nbmodes(Built &b, const std::vector<double> &allpos) {
  WorkSpace &ws = *b.ws;
  set_pos(ws, allpos);
  dump_nb_case(b, "nbfs_", true, false, false, 1.0, false);   // the FF_NonBonded default
  dump_nb_case(b, "nbes_", false, true, false, 1.0, false);
  dump_nb_case(b, "nbnorm_", false, false, false, 1.0, false);
  dump_nb_case(b, "nbddd_", true, false, true, 1.0, false);   // DDDielectric: not consulted by calcForces
  dump_nb_case(b, "nbdiel4_", false, false, false, 4.0, false);
  dump_nb_case(b, "nbvdwcor_", true, false, false, 1.0, true);
  // the GB component with FastMode off, with FF_Bonded, and alone
  b.gb->FastMode = false;
  b.ff->ensuresetup(ws);
  ws.nlist().calcNewList();
  b.ff->calcForces();
  put_d("gbslow_f_total", get_f(ws), shp(ws.nAtoms(), 3));
  put_d("gbslow_ene_total", ene_vec(ws.ene));
  put_d("gbslow_born", born(b));
  ws.zeroForces();
  b.gb->calcForces();
  put_d("gbslow_f_gb", get_f(ws), shp(ws.nAtoms(), 3));
  std::vector<double> e = ene_vec(ws.ene);
  e.push_back(b.gb->epot_pol);
  e.push_back(b.gb->epot_pol_cross);
  e.push_back(b.gb->epot_pol_self);
  put_d("gbslow_ene_gb", e);
  b.gb->FastMode = true;
}

static double now() {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static void usage() {
  fprintf(stderr,
          "ref_driver build --out DIR --nres N[,N..] --seed S [--cutoff R] "
          "[--inner R] [--grid NX,SPACING] [--premin STEPS] [--param F] "
          "[--md STEPS] [--min STEPS] [--slowmode] [--trials K --trial-sigma DEG] [--nbmodes] [--topo-only]\n"
          "          [--lcpo-asp KCAL_PER_A2 --lcpo UPDATESASA[,STEPS[,DENSE]]]\n"
          "ref_driver time --in DIR --cutoff R --inner R --steps K "
          "[--warmup W] [--nlist-every M] [--param F] [--drift] [--fric 1/s]\n"
          "ref_driver evals --in DIR --cutoff R --inner R --steps K [--warmup W] [--param F]\n"
          "ref_driver replay --in DIR --out DIR --cutoff R --inner R [--md STEPS] [--min STEPS] "
          "[--steps K] [--param F]\n");
  exit(1);
}

static std::vector<int> parse_ints(const char *s) {
  std::vector<int> v;
  const char *p = s;
  while (*p) {
    v.push_back(atoi(p));
    while (*p && *p != ',') p++;
    if (*p == ',') p++;
  }
  return v;
}

int main(int argc, char **argv) {
  if (argc < 2) usage();
  std::string mode = argv[1];
  Settings st;
  std::vector<int> nres;
  uint64_t seed = 0;
  int premin = 500, mdsteps = 0, minsteps = 0, steps = 10, warmup = 1, ntrials = 0;
  double trial_sigma_deg = 15.0;
  double lcpo_asp = 0.0;
  int lcpo_update = 5, lcpo_steps = 0, lcpo_dense = 1;
  int nlist_every = 10;
  bool drift = false;
  bool nbmodes = false;
  bool topo_only = false;
  double fric = 1e12;
  int gridx = 0;
  double spacing = 25.0;
  std::string in;
  bool inner_given = false;
  for (int a = 2; a < argc; a++) {
    std::string k = argv[a];
    const char *v = a + 1 < argc ? argv[a + 1] : "";
    if (k == "--out") { g_out = v; a++; }
    else if (k == "--in") { in = v; a++; }
    else if (k == "--nres") { nres = parse_ints(v); a++; }
    else if (k == "--seed") { seed = strtoull(v, NULL, 10); a++; }
    else if (k == "--cutoff") { st.cutoff = atof(v); a++; }
    else if (k == "--inner") { st.inner = atof(v); inner_given = true; a++; }
    else if (k == "--premin") { premin = atoi(v); a++; }
    else if (k == "--md") { mdsteps = atoi(v); a++; }
    else if (k == "--min") { minsteps = atoi(v); a++; }
    else if (k == "--trials") { ntrials = atoi(v); a++; }
    else if (k == "--trial-sigma") { trial_sigma_deg = atof(v); a++; }
    else if (k == "--steps") { steps = atoi(v); a++; }
    else if (k == "--warmup") { warmup = atoi(v); a++; }
    else if (k == "--nlist-every") { nlist_every = atoi(v); a++; }
    else if (k == "--drift") { drift = true; }
    else if (k == "--nbmodes") { nbmodes = true; }
    else if (k == "--topo-only") { topo_only = true; }
    else if (k == "--fric") { fric = atof(v); a++; }
    else if (k == "--param") { st.param = v; a++; }
    else if (k == "--slowmode") { st.fastmode = false; }
    else if (k == "--lcpo") {
      std::vector<int> g = parse_ints(v);
      lcpo_update = g[0];
      if (g.size() > 1) lcpo_steps = g[1];
      if (g.size() > 2) lcpo_dense = g[2];
      a++;
    } else if (k == "--lcpo-asp") { lcpo_asp = atof(v); a++; }
    else if (k == "--grid") {
      std::vector<int> g = parse_ints(v);
      gridx = g[0];
      if (g.size() > 1) spacing = g[1];
      a++;
    } else usage();
  }
  if (!inner_given) st.inner = st.cutoff - 3.0;
  st.vdwcut = st.cutoff;
  st.vdwinner = st.inner;

  FFParamSet *ffps = new FFParamSet();
  ffps->readLib(st.param);

  if (mode == "build") {
    if (g_out.empty() || nres.empty()) usage();
    mkdir(g_out.c_str(), 0755);
    std::vector<std::string> seqs;
    for (size_t k = 0; k < nres.size(); k++)
      seqs.push_back(random_sequence(seed * 1000003ULL + k, nres[k]));
    // pre-minimise each chain alone (12 A cutoff), then place
    std::vector<double> allpos;
    for (size_t k = 0; k < seqs.size(); k++) {
      Settings sm = st;
      sm.cutoff = 12;
      sm.inner = 9;
      sm.vdwcut = 12;
      sm.vdwinner = 9;
      sm.fastmode = true;
      std::vector<std::string> one(1, seqs[k]);
      Built c = make_ws(ffps, one, sm);
      if (premin > 0) preminimise(c, premin);
      std::vector<double> p = get_pos(*c.ws);
      if (gridx > 0) {
        int gx = k % gridx, gy = k / gridx;
        place_chain(p, gx * spacing, gy * spacing);
      }
      allpos.insert(allpos.end(), p.begin(), p.end());
    }
    Built b = make_ws(ffps, seqs, st);
    set_pos(*b.ws, allpos);
    b.ff->ensuresetup(*b.ws);
    // meta
    {
      std::string path = g_out + "/meta.txt";
      FILE *f = fopen(path.c_str(), "w");
      fprintf(f, "natoms %zu\ncutoff %.17g\ninner %.17g\nvdwcut %.17g\nvdwinner %.17g\n",
              b.ws->nAtoms(), st.cutoff, st.inner, st.vdwcut, st.vdwinner);
      fprintf(f, "param %s\nseed %llu\npremin %d\nfastmode %d\n", st.param.c_str(),
              (unsigned long long)seed, premin, (int)st.fastmode);
      fprintf(f, "gridx %d\nspacing %.17g\n", gridx, spacing);
      for (size_t k = 0; k < seqs.size(); k++) fprintf(f, "chain %s\n", seqs[k].c_str());
      fclose(f);
    }
    put_d("pos", allpos, shp(b.ws->nAtoms(), 3));
    dump_topology(b, st);
    if (topo_only) {  // coordinates and topology only (no reference results)
      printf("built %zu atoms\n", b.ws->nAtoms());
      return 0;
    }
    dump_single_point(b, "");
    if (ntrials > 0) dump_trials(b, allpos, ntrials, trial_sigma_deg * 3.14159265358979323846 / 180.0, seed);
    if (minsteps > 0) {
      set_pos(*b.ws, allpos);
      dump_minimise(b, Minimisation::SteepestDescent, minsteps, "minsd_");
      set_pos(*b.ws, allpos);
      dump_minimise(b, Minimisation::ConjugateGradients, minsteps, "mincg_");
    }
    if (mdsteps > 0) {
      set_pos(*b.ws, allpos);
      dump_md_steps(b, MolecularDynamics::Langevin, mdsteps, 1e12, "mdlv_");
      set_pos(*b.ws, allpos);
      dump_md_steps(b, MolecularDynamics::VelocityVerlet, mdsteps, 1e12, "mdvv_");
      set_pos(*b.ws, allpos);
      dump_md_steps(b, MolecularDynamics::Beeman, mdsteps, 1e12, "mdbm_");
    }
    if (lcpo_asp != 0.0) dump_lcpo(b, allpos, lcpo_asp, lcpo_update, lcpo_steps, lcpo_dense != 0);
    if (nbmodes) dump_nbmodes(b, allpos);
    printf("built %zu atoms\n", b.ws->nAtoms());
    return 0;
  }

  if (mode == "replay") {
    if (g_out.empty() || in.empty()) usage();
    mkdir(g_out.c_str(), 0755);
    std::vector<std::string> seqs;
    {
      std::string path = in + "/meta.txt";
      FILE *f = fopen(path.c_str(), "r");
      if (!f) { fprintf(stderr, "no %s\n", path.c_str()); return 2; }
      char key[64], val[4096];
      while (fscanf(f, "%63s %4095s", key, val) == 2)
        if (std::string(key) == "chain") seqs.push_back(val);
      fclose(f);
    }
    size_t n0;
    std::vector<double> pos = npy_read_d(in + "/pos.npy", &n0);
    Built b = make_ws(ffps, seqs, st);
    if (b.ws->nAtoms() != n0) { fprintf(stderr, "atom count mismatch\n"); return 2; }
    set_pos(*b.ws, pos);
    b.ff->ensuresetup(*b.ws);
    dump_single_point(b, "");
    if (mdsteps > 0) {
      set_pos(*b.ws, pos);
      dump_md_steps(b, MolecularDynamics::Langevin, mdsteps, 1e12, "mdlv_");
      set_pos(*b.ws, pos);
      dump_md_steps(b, MolecularDynamics::VelocityVerlet, mdsteps, 1e12, "mdvv_");
    }
    if (minsteps > 0) {
      set_pos(*b.ws, pos);
      dump_minimise(b, Minimisation::SteepestDescent, minsteps, "minsd_");
      set_pos(*b.ws, pos);
      dump_minimise(b, Minimisation::ConjugateGradients, minsteps, "mincg_");
    }
    if (lcpo_asp != 0.0) {
      // the whole forcefield with the LCPO term: a single point at step 0,
      // velocity-Verlet and steepest-descent steps (as dump_lcpo records
      // them for the reference's own component)
      LcpoComponent *sasa = new LcpoComponent(*b.ws);
      sasa->GlobalASP = lcpo_asp;
      sasa->UpdateSasa = lcpo_update;
      b.ff->add(*sasa);
      b.ff->ensuresetup(*b.ws);
      set_pos(*b.ws, pos);
      b.ws->Step = 0;
      b.ws->nlist().calcNewList();
      b.ff->calcForces();
      std::vector<double> e = ene_vec(b.ws->ene);
      e.push_back(b.ws->ene.epot_surf);
      put_d("lcpo_f_total", get_f(*b.ws), shp(b.ws->nAtoms(), 3));
      put_d("lcpo_ene_total", e);
      if (lcpo_steps > 0) {
        set_pos(*b.ws, pos);
        dump_md_steps(b, MolecularDynamics::VelocityVerlet, lcpo_steps, 1e12, "lcpo_mdvv_");
        set_pos(*b.ws, pos);
        b.ws->Step = 0;
        dump_minimise(b, Minimisation::SteepestDescent, lcpo_steps, "lcpo_minsd_");
      }
      printf("replayed %zu atoms\n", b.ws->nAtoms());
      return 0;
    }
    if (steps > 0) {
      // the reference's own protocol loop (md.cpp:202-267) for `steps`
      // Langevin steps, list every 10, velocities drawn by the reference
      set_pos(*b.ws, pos);
      MolecularDynamics md(*b.ff);
      md.Integrator = MolecularDynamics::Langevin;
      md.Timestep = 1e-15;
      md.FricCoeff = 1e12;
      md.Steps = steps;
      md.UpdateNList = nlist_every;
      md.UpdateScr = 0;
      md.OutputLevel = Verbosity::Silent;
      srand(4242);
      md.setInitialSpeeds(300.0);
      int taken = md.runcore();
      put_d("proto_md_x", get_pos(*b.ws), shp(b.ws->nAtoms(), 3));
      std::vector<double> r = ene_vec(b.ws->ene);
      r.push_back(b.ws->ene.ekin);
      r.push_back(taken);
      put_d("proto_md_ene", r);
    }
    printf("replayed %zu atoms\n", b.ws->nAtoms());
    return 0;
  }

  if (mode == "evals") {
    // single-point evaluations as the batched trial scoring does them:
    // NeighbourList::calcNewList + Forcefield::calcForces, `steps` times
    // after `warmup` (the CPU baseline of the batched evaluations)
    std::vector<std::string> seqs;
    {
      std::string path = in + "/meta.txt";
      FILE *f = fopen(path.c_str(), "r");
      if (!f) { fprintf(stderr, "no %s\n", path.c_str()); return 2; }
      char key[64], val[4096];
      while (fscanf(f, "%63s %4095s", key, val) == 2)
        if (std::string(key) == "chain") seqs.push_back(val);
      fclose(f);
    }
    size_t n0;
    std::vector<double> pos = npy_read_d(in + "/pos.npy", &n0);
    Built b = make_ws(ffps, seqs, st);
    if (b.ws->nAtoms() != n0) { fprintf(stderr, "atom count mismatch\n"); return 2; }
    set_pos(*b.ws, pos);
    b.ff->ensuresetup(*b.ws);
    double t0 = 0, e = 0;
    for (int s = 0; s < warmup + steps; s++) {
      if (s == warmup) t0 = now();
      b.ws->nlist().calcNewList();
      b.ff->calcForces();
      e += b.ws->ene.epot;
    }
    double dt = now() - t0;
    printf("{\"evals\": %d, \"seconds\": %.6f, \"natoms\": %zu, \"epot\": %.9g}\n", steps, dt,
           b.ws->nAtoms(), e);
    return 0;
  }

  if (mode == "time") {
    // rebuild the topology from the recorded chains, load coordinates
    std::vector<std::string> seqs;
    {
      std::string path = in + "/meta.txt";
      FILE *f = fopen(path.c_str(), "r");
      if (!f) { fprintf(stderr, "no %s\n", path.c_str()); return 2; }
      char key[64], val[4096];
      while (fscanf(f, "%63s %4095s", key, val) == 2)
        if (std::string(key) == "chain") seqs.push_back(val);
      fclose(f);
    }
    size_t n0;
    std::vector<double> pos = npy_read_d(in + "/pos.npy", &n0);
    Built b = make_ws(ffps, seqs, st);
    if (b.ws->nAtoms() != n0) { fprintf(stderr, "atom count mismatch\n"); return 2; }
    set_pos(*b.ws, pos);
    b.ff->ensuresetup(*b.ws);
    MolecularDynamics md(*b.ff);
    md.Integrator = MolecularDynamics::Langevin;
    md.Timestep = 1e-15;
    md.FricCoeff = fric;
    md.Steps = warmup + steps;
    md.UpdateNList = nlist_every;
    md.UpdateScr = 0;
    md.OutputLevel = Verbosity::Silent;
    srand(1);
    md.setInitialSpeeds(300.0);
    // with --drift: MolecularDynamics::run_core's total-energy drift
    // (md.cpp:206, 231-240, 182-189): etot sampled every max(1, Steps/1000)
    // steps after step 50, least-squares slope in kcal/mol per 1000 steps
    const int total = warmup + steps;
    const int driftfreq = std::max(1, total / 1000);
    std::vector<double> dx, dy;
    double t0 = 0;
    for (int s = 0; s < total; s++) {
      if (s == warmup) t0 = now();
      md.Step = s;
      b.ws->Step = s;
      md.refreshNeighborList();
      b.ff->calcForces();
      md.assertStability();
      md.applyForces();
      if (drift && s > 50 && s % driftfreq == 0) {
        dx.push_back(s);
        dy.push_back((b.ws->ene.epot + b.ws->ene.ekin) * PhysicsConst::J2kcal * PhysicsConst::Na);
      }
    }
    double dt = now() - t0;
    if (drift && dx.size() > 1) {
      double da = 0, db = 0, dR = 0;
      Maths::leastSquaresFit(dx, dy, da, db, dR);
      printf("{\"steps\": %d, \"seconds\": %.6f, \"natoms\": %zu, \"drift_kcal_per_1000\": %.9g}\n", steps,
             dt, b.ws->nAtoms(), 1000.0 * db);
    } else {
      printf("{\"steps\": %d, \"seconds\": %.6f, \"natoms\": %zu}\n", steps, dt, b.ws->nAtoms());
    }
    return 0;
  }
  usage();
  return 0;
}
