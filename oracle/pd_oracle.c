/* CPU restatement of the reference's GB/SA energy-force hot path
 * (JonnyWideFoot/pd.arcus src/mmlib) -- TEST ORACLE ONLY, never on the
 * product path.  Parity with the reference is pinned against outputs of the
 * reference library itself (compiled from source, oracle/Makefile) in
 * tests/test_oracle_golden.py.  Built with -O2 -ffp-contract=off and no
 * fast-math, like the reference's golden build, and with the reference's
 * operation order, so most results agree to the last bit.
 */
#include "pd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- constants
 * forcefield.cpp:18-38 and maths/maths.cpp:6-8, same expressions. */
static const double kPI = 3.14159265358979323846;
static double c_kcal2J, c_J2kcal, c_Na, c_kB, c_Angstrom, c_econv,
    c_econv_joule, c_halfeconv, c_halfeconv_joule;
static int c_init = 0;
static void init_constants(void) {
  if (c_init) return;
  double e_charge = 1.60217645E-19;
  double sqr_e_charge = e_charge * e_charge;
  double e0 = 8.854187817E-12;
  double four_pi = 3.14159265358979323846 * 4.0;
  double _4pi_e0 = four_pi * e0;
  c_kcal2J = 4184.0;
  c_J2kcal = 1.0 / c_kcal2J;
  c_Na = 6.0221418E23;
  c_kB = 1.38065E-23;
  c_Angstrom = 1E-10;
  c_econv = (c_J2kcal * c_Na * sqr_e_charge) / (_4pi_e0 * c_Angstrom);
  c_halfeconv = c_econv * 0.5;
  c_econv_joule = (sqr_e_charge) / (_4pi_e0 * c_Angstrom);
  c_halfeconv_joule = c_econv_joule * 0.5;
  c_init = 1;
}

void pdo_constants(double out[8]) {
  init_constants();
  out[0] = c_kcal2J;
  out[1] = c_J2kcal;
  out[2] = c_Na;
  out[3] = c_kB;
  out[4] = c_Angstrom;
  out[5] = c_econv;
  out[6] = c_econv_joule;
  out[7] = c_halfeconv;
}

static inline double sqr(double x) { return x * x; }
static inline double cube(double x) { return x * x * x; }

/* ---------------------------------------------------------------- bond order
 * bondorder.cpp:77-195: band width from 1-2/1-3/1-4 partners in adjacent
 * residues, band filled 1-4 then 1-3 then 1-2 (later writes win), partners
 * beyond the band kept in a sparse per-atom list. */
int pdo_bondorder(int n, const int *ir, const int *c12p, const int *c12i,
                  const int *c13p, const int *c13i, const int *c14p,
                  const int *c14i, int8_t *band, long band_cap, int *off,
                  int off_cap, int *n_off) {
  const int *ptrs[3] = {c12p, c13p, c14p};
  const int *idxs[3] = {c12i, c13i, c14i};
  int mid = 0;
  for (int i = 0; i < n; i++)
    for (int l = 0; l < 3; l++)
      for (int k = ptrs[l][i]; k < ptrs[l][i + 1]; k++) {
        int lookup = idxs[l][k];
        int d = abs(i - lookup);
        int rd = abs(ir[i] - ir[lookup]);
        if (rd > 1) continue;
        if (d > mid) mid = d;
      }
  mid += 1;
  long need = (long)mid * (n - 1);
  if (need > band_cap) return -1;
  for (long k = 0; k < need; k++) band[k] = 7;
  /* sparse store: per atom i (in order of first appearance) its partners */
  int noff = 0;
  /* order of m_LongBondOrder: atoms appended when first needed; partners
   * appended in calcOrder call order (14, 13, 12) per atom i. */
  int *first_slot = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++) first_slot[i] = -1;
  /* collect per-atom partner lists in a temporary array, then emit in the
   * order atoms were first registered */
  int *tmp = (int *)malloc(sizeof(int) * 3 * (off_cap > 0 ? off_cap : 1));
  int *order_atoms = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int natoms_sparse = 0;
  int ntmp = 0;
  const int orders[3] = {3, 2, 1};
  const int lists[3] = {2, 1, 0}; /* 14, 13, 12 */
  for (int i = 0; i < n; i++) {
    for (int t = 0; t < 3; t++) {
      int l = lists[t];
      for (int k = ptrs[l][i]; k < ptrs[l][i + 1]; k++) {
        int j = idxs[l][k];
        if (j <= i) continue;
        int delta = j - i;
        int order = orders[t] < 7 ? orders[t] : 7;
        if (delta > mid) {
          if (first_slot[i] < 0) {
            first_slot[i] = natoms_sparse;
            order_atoms[natoms_sparse++] = i;
          }
          if (ntmp >= off_cap) {
            free(first_slot);
            free(tmp);
            free(order_atoms);
            return -1;
          }
          tmp[3 * ntmp] = i;
          tmp[3 * ntmp + 1] = j;
          tmp[3 * ntmp + 2] = order;
          ntmp++;
        } else {
          band[(long)i * mid + (delta - 1)] = (int8_t)order;
        }
      }
    }
  }
  for (int s = 0; s < natoms_sparse; s++) {
    int a = order_atoms[s];
    for (int k = 0; k < ntmp; k++)
      if (tmp[3 * k] == a) {
        off[3 * noff] = tmp[3 * k];
        off[3 * noff + 1] = tmp[3 * k + 1];
        off[3 * noff + 2] = tmp[3 * k + 2];
        noff++;
      }
  }
  *n_off = noff;
  free(first_slot);
  free(tmp);
  free(order_atoms);
  return mid;
}

/* ---------------------------------------------------------------- list
 * neighbourlist.cpp:230-316 (InfiniteSpace) and :162-203 (off-diagonal
 * bond-order correction). */
long pdo_nlist(int n, const double *pos, double cutoff, double padding,
               int shadow, int mid, const int8_t *band, int n_off,
               const int *off, int *ptr, int *data, long cap) {
  double lim = sqr(cutoff + padding);
  long cnt = 0;
  for (int i = 0; i < n; i++) {
    ptr[i] = (int)cnt;
    int limit = shadow ? n : i;
    for (int j = 0; j < limit; j++) {
      double dx = pos[3 * j] - pos[3 * i];
      double dy = pos[3 * j + 1] - pos[3 * i + 1];
      double dz = pos[3 * j + 2] - pos[3 * i + 2];
      double d2 = dx * dx + dy * dy + dz * dz;
      if (d2 > lim) continue;
      int bo = 7;
      if (abs(j - i) < mid) {
        if (j > i)
          bo = band[(long)i * mid + (j - i - 1)];
        else
          bo = band[(long)j * mid + (i - j - 1)];
        if (j == i) continue;
      }
      if (cnt >= cap) return -1;
      data[cnt++] = (j & 0x00FFFFFF) | ((bo & 7) << 24);
    }
  }
  ptr[n] = (int)cnt;
  for (int p = 0; p < n_off; p++) {
    int a = off[3 * p], pj = off[3 * p + 1], order = off[3 * p + 2];
    if (shadow || a > pj)
      for (int k = ptr[a]; k < ptr[a + 1]; k++)
        if ((data[k] & 0x00FFFFFF) == pj) {
          data[k] &= (int)0xF8FFFFFF;
          data[k] |= (order & 7) << 24;
          break;
        }
    if (shadow || a < pj)
      for (int k = ptr[pj]; k < ptr[pj + 1]; k++)
        if ((data[k] & 0x00FFFFFF) == a) {
          data[k] &= (int)0xF8FFFFFF;
          data[k] |= (order & 7) << 24;
          break;
        }
  }
  return cnt;
}

/* ---------------------------------------------------------------- GB setup
 * gbff.cpp:307-381. */
void pdo_gb_fixed_terms(int n, const double *gbr, const int *c12p,
                        const int *c12i, const double *c12d, const int *c13p,
                        const int *c13i, const double *c13d,
                        const pdo_params *p, double *vj, double *terms123) {
  const double FourPI = 4.0 * kPI;
  for (int j = 0; j < n; j++) {
    double Rj = gbr[j];
    if (Rj <= 0.01) Rj = 1.15;
    vj[j] = FourPI * Rj * Rj * Rj / 3;
    for (int nk = c12p[j]; nk < c12p[j + 1]; nk++) {
      int k = c12i[nk];
      double Rk = gbr[k];
      if (Rk <= 0.01) Rk = 1.15;
      double rjk = 1.01 * c12d[nk];
      double hjk = Rj * (1.0 + (sqr(Rk) - sqr(Rj) - sqr(rjk)) / (2.0 * Rj * rjk));
      vj[j] -= kPI * sqr(hjk) * (3 * Rj - hjk) / 3;
    }
    if (vj[j] < 0) vj[j] = 0;
  }
  for (int i = 0; i < n; i++) {
    double Rj = gbr[i];
    if (Rj <= 0.01) Rj = 1.15;
    double term1 = -166.0 / (Rj + p->diel_offset + p->P1);
    double term2 = 0;
    for (int nj = c12p[i]; nj < c12p[i + 1]; nj++) {
      int j = c12i[nj];
      double rij = c12d[nj];
      term2 += p->P2 * vj[j] / (sqr(rij) * sqr(rij));
    }
    double term3 = 0;
    for (int nj = c13p[i]; nj < c13p[i + 1]; nj++) {
      int j = c13i[nj];
      double rij = c13d[nj];
      term3 += p->P3 * vj[j] / (sqr(rij) * sqr(rij));
    }
    terms123[i] = term1 + term2 + term3;
  }
}

/* ---------------------------------------------------------------- Born radii
 * gbff.cpp:415-466. */
void pdo_born_radii(int n, const double *pos, const int *ptr, const int *data,
                    const double *gbr, const double *vj,
                    const double *terms123, const pdo_params *p,
                    double *born) {
  init_constants();
  double invP5 = 1 / p->P5;
  for (int i = 0; i < n; i++) {
    double Ri = gbr[i];
    double Gpol = terms123[i];
    for (int nj = ptr[i]; nj < ptr[i + 1]; nj++) {
      int j = data[nj] & 0x00FFFFFF;
      double g = pos[3 * i] - pos[3 * j];
      double h = pos[3 * i + 1] - pos[3 * j + 1];
      double jj = pos[3 * i + 2] - pos[3 * j + 2];
      double Dist_ij = g * g + h * h + jj * jj;
      if (Dist_ij > sqr(p->still_cutoff)) continue;
      if (((data[nj] >> 24) & 7) <= 2) continue;
      double Rj = gbr[j];
      double rdivR = Dist_ij / sqr((Ri + Rj));
      double CCF;
      if (rdivR > invP5)
        CCF = 1.0;
      else
        CCF = sqr(0.5 - 0.5 * cos((rdivR * p->P5 * kPI)));
      Gpol += p->P4 * vj[j] * CCF / (sqr(Dist_ij));
    }
    born[i] = -c_halfeconv / Gpol + p->born_offset;
  }
}

/* ---------------------------------------------------------------- GB forces
 * gbff.cpp:1449-1818 (FastMode: GB + vacuum LJ/Coulomb in one pass, then the
 * Born-radius chain rule over the full list). */
void pdo_gb_forces(int n, const double *pos, const int *ptr, const int *data,
                   const double *q, const double *radius, const double *eps,
                   const double *gbr, const double *vj, const double *born,
                   const pdo_params *p, double *f, double *ene,
                   double *atom_epot, double *deda_out) {
  init_constants();
  double sqrcutoff = sqr(p->cutoff);
  double Swidth = p->cutoff - p->inner_cutoff;
  double invSwidth = 1.0 / Swidth;
  double vdwSwidth = p->vdw_cutoff - p->vdw_inner_cutoff;
  double vdwinvSwidth = 1.0 / vdwSwidth;
  double invdielectric = 1 / p->diel_solute;
  double invsolventdielectric = 1 / p->diel_solvent;
  double premul = -c_halfeconv_joule * (1 / p->diel_solute - 1 / p->diel_solvent);
  double e_vdw = 0, e_elec = 0, e_total = 0;
  double epot_pol = 0, epot_pol_self = 0, epot_pol_cross = 0;
  double *dedi = (double *)calloc((size_t)3 * n + 1, sizeof(double));
  double *deda = (double *)calloc((size_t)n + 1, sizeof(double));
  double *aepot = atom_epot;
  if (aepot) memset(aepot, 0, sizeof(double) * n);

  for (int i = 0; i < n; i++) {
    double ai = born[i];
    double atomix = pos[3 * i], atomiy = pos[3 * i + 1], atomiz = pos[3 * i + 2];
    double dedai = 0;
    double atomi_radius = radius[i];
    double atomi_epsilon = eps[i];
    double qi = q[i];
    for (int nj = ptr[i]; nj < ptr[i + 1]; nj++) {
      int j = data[nj] & 0x00FFFFFF;
      if (j > i) break;
      int typej = (data[nj] >> 24) & 7;
      double aj = born[j];
      double qiqj = qi * q[j];
      double dddx = (double)(atomix - pos[3 * j]);
      double dddy = (double)(atomiy - pos[3 * j + 1]);
      double dddz = (double)(atomiz - pos[3 * j + 2]);
      double srij = sqr(dddx) + sqr(dddy) + sqr(dddz);
      if (srij > sqrcutoff) continue;
      double Dist_ij = sqrt(srij);
      double invdistij = 1 / Dist_ij;
      double aiaj = ai * aj;
      double uGB = -srij * 0.25 / aiaj;
      double pair_elec14scaling = 1.0;
      if (typej == 3) pair_elec14scaling = p->elec14;
      double elec_potential = 0, elec_force = 0;
      double S, dSdd, dedx, dedy, dedz;
      if (uGB > p->exp_thresh) {
        double tGB = exp(uGB);
        double mGB = tGB * aiaj;
        double lGB = 1 / (srij + mGB);
        double fGB = sqrt(lGB);
        double epol = premul * qiqj * fGB;
        double dedr = -epol * (Dist_ij - 0.25 * Dist_ij * tGB) * lGB;
        double dedalpha = -epol * tGB * (1.0 - uGB) * lGB;
        if (typej >= 3) {
          elec_potential = (double)c_econv_joule * invdielectric * pair_elec14scaling * qiqj * invdistij;
          elec_force = -elec_potential * invdistij;
        }
        if (Dist_ij >= p->inner_cutoff) {
          S = (1.0 - sqr(invSwidth * (Dist_ij - p->inner_cutoff)));
          dSdd = -4.0 * sqr(invSwidth) * (Dist_ij - p->inner_cutoff) * S;
          S = sqr(S);
          elec_force = S * elec_force + elec_potential * dSdd;
          elec_potential *= S;
          dedr = S * dedr + dSdd * epol;
          dedalpha *= S;
          epol *= S;
        }
        dedr *= 2 * invdistij;
        dedx = dedr * dddx;
        dedy = dedr * dddy;
        dedz = dedr * dddz;
        epot_pol += epol;
        epot_pol += epol;
        epot_pol_cross += epol;
        epot_pol_cross += epol;
        if (aepot) {
          aepot[i] += epol;
          aepot[j] += epol;
        }
        dedi[3 * i] += dedx;
        dedi[3 * i + 1] += dedy;
        dedi[3 * i + 2] += dedz;
        dedi[3 * j] -= dedx;
        dedi[3 * j + 1] -= dedy;
        dedi[3 * j + 2] -= dedz;
        dedai += dedalpha * aj;
        deda[j] += dedalpha * ai;
      } else {
        if (typej >= 3) {
          elec_potential = c_econv_joule * invsolventdielectric * pair_elec14scaling * qiqj * invdistij;
          elec_force = -elec_potential * invdistij;
          if (Dist_ij >= p->inner_cutoff) {
            S = (1.0 - sqr(invSwidth * (Dist_ij - p->inner_cutoff)));
            dSdd = -4.0 * sqr(invSwidth) * (Dist_ij - p->inner_cutoff) * S;
            S = sqr(S);
            elec_force = S * elec_force + elec_potential * dSdd;
            elec_potential *= S;
          }
        }
      }
      if (typej >= 3) {
        double pair_vdw14scaling = 1.0;
        if (typej == 3) pair_vdw14scaling = p->vdw14;
        double vdw_force = 0, vdw_potential = 0;
        if (Dist_ij < p->vdw_cutoff) {
          double radiusij = sqr(invdistij * (atomi_radius + radius[j]));
          double epsilon = pair_vdw14scaling * atomi_epsilon * eps[j];
          double B = cube(radiusij);
          double A = sqr(B);
          vdw_potential = (2.0 * epsilon) * (0.5 * A - B);
          vdw_force = -(12.0 * epsilon * invdistij) * (A - B);
          if (Dist_ij > p->vdw_inner_cutoff) {
            double vdwS = (1.0 - sqr(vdwinvSwidth * (Dist_ij - p->vdw_inner_cutoff)));
            double vdwdSdd = -4.0 * sqr(vdwinvSwidth) * (Dist_ij - p->vdw_inner_cutoff) * vdwS;
            vdwS = sqr(vdwS);
            vdw_force = vdwS * vdw_force + vdw_potential * vdwdSdd;
            vdw_potential *= vdwS;
          }
          e_total += vdw_potential;
          e_vdw += vdw_potential;
          if (aepot) {
            aepot[i] += vdw_potential * 0.5;
            aepot[j] += vdw_potential * 0.5;
          }
        }
        e_total += elec_potential;
        e_elec += elec_potential;
        if (aepot) {
          aepot[i] += elec_potential * 0.5;
          aepot[j] += elec_potential * 0.5;
        }
        double force_magnitude = 0;
        force_magnitude += vdw_force;
        force_magnitude += elec_force;
        force_magnitude *= invdistij;
        dedx = force_magnitude * dddx;
        dedy = force_magnitude * dddy;
        dedz = force_magnitude * dddz;
        dedi[3 * i] += dedx;
        dedi[3 * i + 1] += dedy;
        dedi[3 * i + 2] += dedz;
        dedi[3 * j] -= dedx;
        dedi[3 * j + 1] -= dedy;
        dedi[3 * j + 2] -= dedz;
      }
    }
    deda[i] += dedai;
    double epol = premul * sqr(qi) / ai;
    epot_pol += epol;
    epot_pol_self += epol;
    if (aepot) aepot[i] += epol;
    deda[i] += -epol / ai;
  }
  e_total += epot_pol;

  /* second part: chain rule through the Born radii (gbff.cpp:1751-1808) */
  double invP5 = 1 / p->P5;
  for (int i = 0; i < n; i++) {
    double Ri = gbr[i];
    double gpi = -sqr(born[i]) / -166.0;
    for (int nj = ptr[i]; nj < ptr[i + 1]; nj++) {
      int j = data[nj] & 0x00FFFFFF;
      double dddx = (pos[3 * j] - pos[3 * i]);
      double dddy = (pos[3 * j + 1] - pos[3 * i + 1]);
      double dddz = (pos[3 * j + 2] - pos[3 * i + 2]);
      double srij = sqr(dddx) + sqr(dddy) + sqr(dddz);
      if (srij > sqr(p->still_cutoff)) continue;
      if (((data[nj] >> 24) & 7) <= 2) continue;
      double Rj = gbr[j];
      double Vj = vj[j];
      double r6 = srij * srij * srij;
      double rdivR = srij / sqr((Ri + Rj));
      double CCF, dCCF;
      if (rdivR > invP5) {
        CCF = 1.0;
        dCCF = 0.0;
      } else {
        double theta = rdivR * p->P5 * kPI;
        double sintheta = sin(theta);
        double costheta = cos(theta);
        double sqrtCCF = 0.5 - 0.5 * costheta;
        CCF = sqr(sqrtCCF);
        dCCF = 2.0 * sqrtCCF * sintheta * theta;
      }
      double dedr = gpi * deda[i] * p->P4 * Vj * (4.0 * CCF - dCCF) / r6;
      double dedx = dedr * dddx;
      double dedy = dedr * dddy;
      double dedz = dedr * dddz;
      dedi[3 * i] += dedx;
      dedi[3 * i + 1] += dedy;
      dedi[3 * i + 2] += dedz;
      dedi[3 * j] -= dedx;
      dedi[3 * j + 1] -= dedy;
      dedi[3 * j + 2] -= dedz;
    }
  }
  for (int i = 0; i < n; i++) {
    double m = (double)-1.0 / (double)(c_Angstrom);
    f[3 * i] += dedi[3 * i] * m;
    f[3 * i + 1] += dedi[3 * i + 1] * m;
    f[3 * i + 2] += dedi[3 * i + 2] * m;
  }
  ene[0] = e_total;
  ene[1] = e_vdw;
  ene[2] = e_elec;
  ene[3] = epot_pol;
  ene[4] = epot_pol_cross;
  ene[5] = epot_pol_self;
  if (deda_out) memcpy(deda_out, deda, sizeof(double) * n);
  free(dedi);
  free(deda);
}

/* ---------------------------------------------------------------- Born energy
 * gbff.cpp:520-579 (energy-only path; no exp-threshold branch). */
double pdo_born_energy(int n, const double *pos, const int *ptr,
                       const int *data, const double *q, const double *born,
                       const pdo_params *p, double *pol) {
  init_constants();
  double Swidth = p->cutoff - p->inner_cutoff;
  double invSwidth = 1 / Swidth;
  double bornpremul = -c_halfeconv_joule * (1 / p->diel_solute - 1 / p->diel_solvent);
  double epot_pol = 0, epot_pol_self = 0, epot_pol_cross = 0;
  for (int i = 0; i < n; i++) {
    double qi = q[i];
    double ai = born[i];
    epot_pol -= sqr(qi) / ai;
    epot_pol_self -= sqr(qi) / ai;
    for (int nj = ptr[i]; nj < ptr[i + 1]; nj++) {
      int j = data[nj] & 0x00FFFFFF;
      if (i > j) continue;
      double g = pos[3 * i] - pos[3 * j];
      double h = pos[3 * i + 1] - pos[3 * j + 1];
      double jj = pos[3 * i + 2] - pos[3 * j + 2];
      double Dist_ij = sqrt(g * g + h * h + jj * jj);
      if (Dist_ij > p->cutoff) continue;
      double S;
      if (Dist_ij < p->inner_cutoff) {
        S = 1.0;
      } else {
        S = (1.0 - sqr(invSwidth * (Dist_ij - p->inner_cutoff)));
        S = sqr(S);
      }
      double srij = sqr(Dist_ij);
      double qj = q[j];
      double aiaj = ai * born[j];
      double epol = 2.0 * S * qi * qj / sqrt(srij + aiaj * exp(-srij * 0.25 / aiaj));
      epot_pol -= epol;
      epot_pol_cross -= epol;
    }
  }
  epot_pol *= -bornpremul;
  epot_pol_cross *= -bornpremul;
  epot_pol_self *= -bornpremul;
  if (pol) {
    pol[0] = epot_pol;
    pol[1] = epot_pol_cross;
    pol[2] = epot_pol_self;
  }
  return epot_pol;
}

/* ---------------------------------------------------------------- LJ + Coulomb
 * FF_NonBonded_CalcForces_T_fast2 (nonbonded.cpp:548-893) with the mode
 * selection of FF_NonBonded::calcForces (nonbonded.cpp:1205-1229): VdW mode
 * EnergySwitch unless DoVdw is off; elec mode Normal, EnergySwitch or
 * ForceSwitch (ForceSwitch wins when both are set), or None; the
 * DDDielectric mode is the Levitt form selected only by an explicit mode
 * (ddd=1 here, as the reference template T_ElecMode_DDDielectric_Levitt). */
void pdo_nonbonded(int n, const double *pos, const int *ptr, const int *data,
                   const double *q, const double *radius, const double *eps,
                   const pdo_params *p, double *f, double *ene) {
  init_constants();
  const double sqrcutoff = sqr(p->cutoff);
  const double sqrinnercutoff = sqr(p->inner_cutoff);
  const double invdielectric = 1.0 / p->dielectric;
  const double Swidth = p->cutoff - p->inner_cutoff;
  const double invSwidth = 1.0 / Swidth;
  const double vdwSwidth = p->vdw_cutoff - p->vdw_inner_cutoff;
  const double vdwinvSwidth = 1.0 / vdwSwidth;
  const double Rc = p->cutoff, Ri = p->inner_cutoff;
  const double sA = 1.0 / cube(sqr(Rc) - sqr(Ri));
  const double sB = -(cube(sqr(Rc)) - 3.0 * sqr(Rc) * sqr(Rc) * sqr(Ri));
  const double sC = 6.0 * sqr(Rc) * sqr(Ri);
  const double sD = -(sqr(Rc) + sqr(Ri));
  const double sE = 2.0 / 5.0;
  const double fswitch_innerV = sA * (sB * (1.0 / Ri) + sC * Ri + sD * cube(Ri) + sE * cube(Ri) * sqr(Ri));
  const double fswitch_cutoffV = sA * (sB * (1.0 / Rc) + sC * Rc + sD * cube(Rc) + sE * cube(Rc) * sqr(Rc));
  double eshift;
  if (Ri < Rc)
    eshift = 1 / Ri + (fswitch_innerV - fswitch_cutoffV);
  else
    eshift = 0;
  int vdwmode = p->do_vdw ? 2 : 0;
  int elecmode = 1;
  if (p->energy_switch) elecmode = 3;
  if (p->force_switch) elecmode = 4;
  if (p->ddd) elecmode = 2;
  if (!p->do_elec) elecmode = 0;
  double tabVdw[8] = {0.0, 0.0, 0.0, p->vdw14, 1.0, 1.0, 1.0, 1.0};
  double tabElec[8] = {0.0, 0.0, 0.0, p->elec14, 1.0, 1.0, 1.0, 1.0};
  double epot = 0, evdw = 0, eelec = 0, vir = 0;
  for (int i = 0; i < n; i++) {
    double atomi_radius = radius[i];
    double atomi_epsilon = eps[i];
    double qi = q[i];
    double fvi[3] = {0, 0, 0};
    for (int nj = ptr[i]; nj < ptr[i + 1]; nj++) {
      int j = data[nj];
      int nbor_type = j >> 24;
      j &= 0x00FFFFFF;
      if (j >= i) break;
      double vdw14scale = tabVdw[nbor_type & 7];
      double elec14scale = tabElec[nbor_type & 7];
      double fv[3] = {pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1],
                      pos[3 * j + 2] - pos[3 * i + 2]};
      fv[0] += 0.0;
      fv[1] += 0.0;
      fv[2] += 0.0; /* basisvector[0] of infinite space is zero */
      double sqrdistij = fv[0] * fv[0] + fv[1] * fv[1] + fv[2] * fv[2];
      if (sqrdistij > sqrcutoff) continue;
      double Dist_ij = sqrt(sqrdistij);
      double invdistij = 1.0 / Dist_ij;
      double vdw_potential = 0, vdw_force = 0, elec_potential = 0, elec_force = 0;
      if (vdwmode > 0) {
        if (Dist_ij < p->vdw_cutoff) {
          double radiusij = atomi_radius + radius[j];
          double epsilon = vdw14scale * atomi_epsilon * eps[j];
          double B = sqr(radiusij * invdistij);
          B *= B * B;
          double A = sqr(B);
          vdw_potential = (2.0 * epsilon) * (0.5 * A - B);
          vdw_force = -(12.0E10 * epsilon * invdistij) * (A - B);
          if (vdwmode == 2) {
            if (Dist_ij > p->vdw_inner_cutoff) {
              double vdwS = (1.0 - sqr(vdwinvSwidth * (Dist_ij - p->vdw_inner_cutoff)));
              double vdwdSdd = -4.0E10 * sqr(vdwinvSwidth) * (Dist_ij - p->vdw_inner_cutoff) * vdwS;
              vdwS = sqr(vdwS);
              vdw_force = vdwS * vdw_force + vdw_potential * vdwdSdd;
              vdw_potential *= vdwS;
            }
          }
        }
      }
      if (elecmode > 0) {
        double qj = q[j];
        if (elecmode == 1) {
          elec_potential = c_econv_joule * invdielectric * elec14scale * (qi * qj) * invdistij;
          elec_force = -elec_potential * invdistij * 1E10;
        }
        if (elecmode == 2) {
          double incdistij = ((p->dielectric + p->ddd_alpha * Dist_ij) * Dist_ij);
          elec_potential = c_econv_joule * elec14scale * (qi * qj) / incdistij;
          elec_force = -elec_potential * (p->dielectric + 2.0 * p->ddd_alpha * Dist_ij) / (incdistij * c_Angstrom);
        }
        if (elecmode == 3) {
          elec_potential = c_econv_joule * invdielectric * elec14scale * (qi * qj) * invdistij;
          elec_force = -elec_potential * invdistij * 1E10;
          if (Dist_ij > p->inner_cutoff) {
            double S = (1.0 - sqr(invSwidth * (Dist_ij - p->inner_cutoff)));
            double dSdd = -4.0E10 * sqr(invSwidth) * (Dist_ij - p->inner_cutoff) * S;
            S = sqr(S);
            elec_force = S * elec_force + elec_potential * dSdd;
            elec_potential *= S;
          }
        }
        if (elecmode == 4) {
          elec_potential = c_econv_joule * invdielectric * elec14scale * (qi * qj);
          if (Dist_ij > p->inner_cutoff) {
            elec_force = -1E10 * elec_potential * sA * sqr(invdistij) * sqr(sqrcutoff - sqrdistij) *
                         (sqrcutoff - 3.0 * sqrinnercutoff + 2.0 * sqrdistij);
            elec_potential *= -(sA * Dist_ij * (sB * sqr(invdistij) + sC + sD * sqrdistij + sE * sqr(sqrdistij)) -
                                fswitch_cutoffV);
          } else {
            elec_force = -1E10 * elec_potential * sqr(invdistij);
            elec_potential *= (invdistij - eshift);
          }
        }
      }
      epot += vdw_potential + elec_potential;
      evdw += vdw_potential;
      eelec += elec_potential;
      double force_magnitude = vdw_force + elec_force;
      vir += Dist_ij * force_magnitude * c_Angstrom;
      double s = invdistij * force_magnitude;
      fv[0] *= s;
      fv[1] *= s;
      fv[2] *= s;
      fvi[0] += fv[0];
      fvi[1] += fv[1];
      fvi[2] += fv[2];
      f[3 * j] -= fv[0];
      f[3 * j + 1] -= fv[1];
      f[3 * j + 2] -= fv[2];
    }
    f[3 * i] += fvi[0];
    f[3 * i + 1] += fvi[1];
    f[3 * i + 2] += fvi[2];
    if (p->vdwcor) {
      double vp = -0.5 * p->vdwcor_density * p->vdwcor_eps / (c_J2kcal * c_Na) * (8.0 / 3.0) * kPI *
                  sqr(p->vdwcor_radius) * sqr(p->vdwcor_radius) * sqr(p->vdwcor_radius) / cube(p->vdwcor_cutoff);
      epot += vp;
      evdw += vp;
    }
  }
  ene[0] = epot;
  ene[1] = evdw;
  ene[2] = eelec;
  ene[3] = vir;
}

/* ---------------------------------------------------------------- bonded */
static void dihedral(const double *pos, const int *idx, int terms,
                     const double *par, double *f, double *epot_out) {
  int ti = idx[0], ta = idx[1], tb = idx[2], tj = idx[3];
  double a[3], b[3], c[3];
  for (int k = 0; k < 3; k++) {
    a[k] = pos[3 * ti + k] - pos[3 * ta + k];
    b[k] = pos[3 * ta + k] - pos[3 * tb + k];
    c[k] = pos[3 * tb + k] - pos[3 * tj + k];
  }
  double fi[3] = {0, 0, 0}, fab[3] = {0, 0, 0}, fj[3] = {0, 0, 0};
  double n1[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  double n2[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  double n3[3] = {b[1] * n1[2] - b[2] * n1[1], b[2] * n1[0] - b[0] * n1[2], b[0] * n1[1] - b[1] * n1[0]};
  double in1 = 1.0 / sqrt(sqr(n1[0]) + sqr(n1[1]) + sqr(n1[2]));
  double in2 = 1.0 / sqrt(sqr(n2[0]) + sqr(n2[1]) + sqr(n2[2]));
  double in3 = 1.0 / sqrt(sqr(n3[0]) + sqr(n3[1]) + sqr(n3[2]));
  double cos_phi = (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]) * in1 * in2;
  double sin_phi = (n3[0] * n2[0] + n3[1] * n2[1] + n3[2] * n2[2]) * in3 * in2;
  n2[0] *= in2;
  n2[1] *= in2;
  n2[2] *= in2;
  double phi = -atan2(sin_phi, cos_phi);
  double dc1[3] = {0, 0, 0}, dc2[3] = {0, 0, 0}, ds3[3] = {0, 0, 0}, ds2[3] = {0, 0, 0};
  if (fabs(sin_phi) > 0.1) {
    n1[0] *= in1;
    n1[1] *= in1;
    n1[2] *= in1;
    for (int k = 0; k < 3; k++) {
      dc1[k] = in1 * (n1[k] * cos_phi - n2[k]);
      dc2[k] = in2 * (n2[k] * cos_phi - n1[k]);
    }
  } else {
    n3[0] *= in3;
    n3[1] *= in3;
    n3[2] *= in3;
    for (int k = 0; k < 3; k++) {
      ds3[k] = in3 * (n3[k] * sin_phi - n2[k]);
      ds2[k] = in2 * (n2[k] * sin_phi - n3[k]);
    }
  }
  double e_this = 0;
  for (int t = 0; t < terms; t++) {
    double k = par[t], nn = par[4 + t], gamma = par[8 + t];
    double epot, dEdphi;
    if (nn > 0) {
      epot = k * (1.0 + cos(nn * phi + gamma));
      dEdphi = -nn * k * sin(nn * phi + gamma);
    } else {
      double diff = phi - gamma;
      if (diff < -kPI)
        diff += 2.0 * kPI;
      else if (diff > kPI)
        diff -= 2.0 * kPI;
      epot = k * sqr(diff);
      dEdphi = 2.0 * k * diff;
    }
    e_this += epot;
    if (fabs(sin_phi) > 0.1) {
      dEdphi /= sin_phi;
      fi[0] += dEdphi * (b[1] * dc1[2] - b[2] * dc1[1]);
      fi[1] += dEdphi * (b[2] * dc1[0] - b[0] * dc1[2]);
      fi[2] += dEdphi * (b[0] * dc1[1] - b[1] * dc1[0]);
      fj[0] += dEdphi * (b[2] * dc2[1] - b[1] * dc2[2]);
      fj[1] += dEdphi * (b[0] * dc2[2] - b[2] * dc2[0]);
      fj[2] += dEdphi * (b[1] * dc2[0] - b[0] * dc2[1]);
      fab[0] += dEdphi * (a[2] * dc1[1] - a[1] * dc1[2] + c[1] * dc2[2] - c[2] * dc2[1]);
      fab[1] += dEdphi * (a[0] * dc1[2] - a[2] * dc1[0] + c[2] * dc2[0] - c[0] * dc2[2]);
      fab[2] += dEdphi * (a[1] * dc1[0] - a[0] * dc1[1] + c[0] * dc2[1] - c[1] * dc2[0]);
    } else {
      dEdphi /= -cos_phi;
      fi[0] += dEdphi * ((b[1] * b[1] + b[2] * b[2]) * ds3[0] - b[0] * b[1] * ds3[1] - b[0] * b[2] * ds3[2]);
      fi[1] += dEdphi * ((b[2] * b[2] + b[0] * b[0]) * ds3[1] - b[1] * b[2] * ds3[2] - b[1] * b[0] * ds3[0]);
      fi[2] += dEdphi * ((b[0] * b[0] + b[1] * b[1]) * ds3[2] - b[2] * b[0] * ds3[0] - b[2] * b[1] * ds3[1]);
      fj[0] += dEdphi * (ds2[1] * b[2] - ds2[2] * b[1]);
      fj[1] += dEdphi * (ds2[2] * b[0] - ds2[0] * b[2]);
      fj[2] += dEdphi * (ds2[0] * b[1] - ds2[1] * b[0]);
      fab[0] += dEdphi * (-(b[1] * a[1] + b[2] * a[2]) * ds3[0] + (2.0 * b[0] * a[1] - a[0] * b[1]) * ds3[1] +
                          (2.0 * b[0] * a[2] - a[0] * b[2]) * ds3[2] + ds2[2] * c[1] - ds2[1] * c[2]);
      fab[1] += dEdphi * (-(b[2] * a[2] + b[0] * a[0]) * ds3[1] + (2.0 * b[1] * a[2] - a[1] * b[2]) * ds3[2] +
                          (2.0 * b[1] * a[0] - a[1] * b[0]) * ds3[0] + ds2[0] * c[2] - ds2[2] * c[0]);
      fab[2] += dEdphi * (-(b[0] * a[0] + b[1] * a[1]) * ds3[2] + (2.0 * b[2] * a[0] - a[2] * b[0]) * ds3[0] +
                          (2.0 * b[2] * a[1] - a[2] * b[1]) * ds3[1] + ds2[1] * c[0] - ds2[0] * c[1]);
    }
  }
  double inv = 1.0 / c_Angstrom;
  for (int k = 0; k < 3; k++) {
    fi[k] *= inv;
    fab[k] *= inv;
    fj[k] *= inv;
  }
  for (int k = 0; k < 3; k++) {
    f[3 * ti + k] += fi[k];
    f[3 * ta + k] += fab[k] - fi[k];
    f[3 * tb + k] += fj[k] - fab[k];
    f[3 * tj + k] -= fj[k];
  }
  *epot_out += e_this;
}

void pdo_bonded(int n, const double *pos, int nb, const int *bij,
                const double *blk, int na, const int *aiaj, const double *akt,
                int nt, const int *tidx, const int *tterms,
                const double *tpar, int ni, const int *iidx,
                const int *iterms, const double *ipar, double *f,
                double *ene) {
  init_constants();
  (void)n;
  double ebond = 0, eangle = 0, etors = 0, eimpr = 0, vir = 0;
  for (int ib = 0; ib < nb; ib++) {
    int i = bij[2 * ib], j = bij[2 * ib + 1];
    double l = blk[2 * ib], k = blk[2 * ib + 1];
    double vb[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1], pos[3 * i + 2] - pos[3 * j + 2]};
    double d = sqrt(vb[0] * vb[0] + vb[1] * vb[1] + vb[2] * vb[2]);
    double fm = 2 * k * (d - l) / c_Angstrom;
    vir += d * fm * c_Angstrom;
    ebond += k * sqr(d - l);
    double s = fm / d;
    for (int c = 0; c < 3; c++) {
      vb[c] *= s;
      f[3 * i + c] -= vb[c];
      f[3 * j + c] += vb[c];
    }
  }
  for (int ib = 0; ib < na; ib++) {
    double k = akt[2 * ib], theta0 = akt[2 * ib + 1];
    if (k == 0) continue;
    int i = aiaj[3 * ib], a = aiaj[3 * ib + 1], j = aiaj[3 * ib + 2];
    double iv[3], jv[3], uiv[3], ujv[3];
    for (int c = 0; c < 3; c++) iv[c] = pos[3 * i + c] - pos[3 * a + c];
    double iv_mag = sqrt(sqr(iv[0]) + sqr(iv[1]) + sqr(iv[2]));
    double inv_iv = 1 / iv_mag;
    for (int c = 0; c < 3; c++) uiv[c] = iv[c] * inv_iv;
    for (int c = 0; c < 3; c++) jv[c] = pos[3 * j + c] - pos[3 * a + c];
    double jv_mag = sqrt(sqr(jv[0]) + sqr(jv[1]) + sqr(jv[2]));
    double inv_jv = 1 / jv_mag;
    for (int c = 0; c < 3; c++) ujv[c] = jv[c] * inv_jv;
    double cos_theta = uiv[0] * ujv[0] + uiv[1] * ujv[1] + uiv[2] * ujv[2];
    double theta = acos(cos_theta);
    double sin_theta = sin(theta);
    eangle += k * sqr(theta - theta0);
    double fm = 2 * k * (theta - theta0) / (c_Angstrom);
    double bn[3];
    for (int c = 0; c < 3; c++) bn[c] = fm * inv_iv * (uiv[c] * cos_theta - ujv[c]) / sin_theta;
    for (int c = 0; c < 3; c++) {
      f[3 * i + c] -= bn[c];
      f[3 * a + c] += bn[c];
    }
    for (int c = 0; c < 3; c++) bn[c] = fm * inv_jv * (ujv[c] * cos_theta - uiv[c]) / sin_theta;
    for (int c = 0; c < 3; c++) {
      f[3 * j + c] -= bn[c];
      f[3 * a + c] += bn[c];
    }
  }
  for (int t = 0; t < nt; t++) dihedral(pos, tidx + 4 * t, tterms[t], tpar + 12 * t, f, &etors);
  for (int t = 0; t < ni; t++) dihedral(pos, iidx + 4 * t, iterms[t], ipar + 12 * t, f, &eimpr);
  ene[0] = ebond;
  ene[1] = eangle;
  ene[2] = etors + eimpr;
  ene[3] = vir;
  ene[4] = ebond + eangle + etors + eimpr;
}

/* ---------------------------------------------------------------- MD steps */
static double kinetic(int n, const double *v, const double *mass) {
  double ekin = 0;
  for (int i = 0; i < n; i++) {
    double mag = sqrt(v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    ekin += (0.5 * mass[i] * sqr(mag));
  }
  return ekin;
}

/* md.cpp:788-838 (the reference adds the half-kick once before the kinetic
 * energy and twice more in the position loop; reproduced as written). */
double pdo_velocity_verlet_step(int n, double *x, double *v, const double *f,
                                const double *mass, double dt) {
  init_constants();
  double t = dt;
  for (int i = 0; i < n; i++) {
    double tinvmass = 0.5 * t / mass[i];
    for (int c = 0; c < 3; c++) v[3 * i + c] += f[3 * i + c] * tinvmass;
  }
  double ekin = kinetic(n, v, mass);
  for (int i = 0; i < n; i++) {
    double tinvmass = 0.5 * t / mass[i];
    double dv[3], dr[3];
    for (int c = 0; c < 3; c++) {
      dv[c] = f[3 * i + c] * tinvmass;
      v[3 * i + c] += dv[c];
    }
    for (int c = 0; c < 3; c++) dr[c] = t * (v[3 * i + c] + dv[c]);
    for (int c = 0; c < 3; c++) {
      dr[c] *= 1 / c_Angstrom;
      x[3 * i + c] += dr[c];
      v[3 * i + c] += dv[c];
    }
  }
  return ekin;
}

/* md.cpp:841-902 (Beeman, the reference's default integrator). */
double pdo_beeman_step(int n, double *x, double *v, const double *f,
                       double *fold, const double *mass, double dt, int step,
                       int steps) {
  init_constants();
  double t = dt;
  if (step > 0)
    for (int i = 0; i < n; i++) {
      double tinvmass = t / (6.0 * mass[i]);
      for (int c = 0; c < 3; c++) v[3 * i + c] += ((2.0) * f[3 * i + c]) * tinvmass;
    }
  double ekin = kinetic(n, v, mass);
  if (step < (steps - 1))
    for (int i = 0; i < n; i++) {
      double tinvmass = t / (6.0 * mass[i]);
      double dr[3], dv[3];
      for (int c = 0; c < 3; c++) {
        dr[c] = t * (v[3 * i + c] + (4.0 * f[3 * i + c] - fold[3 * i + c]) * tinvmass);
        dr[c] *= 1 / c_Angstrom;
        dv[c] = (5.0 * f[3 * i + c] - fold[3 * i + c]) * tinvmass;
      }
      for (int c = 0; c < 3; c++) {
        x[3 * i + c] += dr[c];
        v[3 * i + c] += dv[c];
        fold[3 * i + c] = f[3 * i + c];
      }
    }
  return ekin;
}

/* md.cpp:906-1042 (Langevin, stochastic on all atoms). */
double pdo_langevin_step(int n, double *x, double *v, const double *f,
                         const double *mass, const double *normals, double dt,
                         double gamma, double temp, int step, int steps) {
  init_constants();
  double t = dt;
  double gammat = gamma * t;
  double gt = gammat;
  double gt2 = gt * gt, gt3 = gt * gt2, gt4 = gt2 * gt2, gt5 = gt2 * gt3;
  double gt6 = gt3 * gt3, gt7 = gt3 * gt4, gt8 = gt4 * gt4, gt9 = gt4 * gt5;
  double c0, c1, c2, varv, varr, crv;
  if (gammat < 0.00001) return pdo_velocity_verlet_step(n, x, v, f, mass, dt);
  if (gammat > 0.05) {
    c0 = exp(-gammat);
    c1 = (1 - c0) / gammat;
    c2 = (1 - c1) / gammat;
    double egammat = exp(-gammat);
    varv = (1.0 - sqr(egammat));
    varr = (2.0 * gammat - 3.0 + (4.0 - egammat) * egammat);
    crv = sqr(1.0 - egammat) / (sqrt(varv * varr));
  } else {
    c0 = 1 - gt + 0.5 * gt2 - gt3 / 6.0 + gt4 / 24.0 - gt5 / 120.0 + gt6 / 720.0 - gt7 / 5040.0 + gt8 / 40320.0 -
         gt9 / 362880.0;
    c1 = 1 - (0.5 * gt - gt2 / 6.0 + gt3 / 24.0 - gt4 / 120.0 + gt5 / 720.0 - gt6 / 5040.0 + gt7 / 40320.0 -
              gt8 / 362880.0);
    c2 = 0.5 - gt / 6.0 + gt2 / 24.0 - gt3 / 120.0 + gt4 / 720.0 - gt5 / 5040.0 + gt6 / 40320.0 - gt7 / 362880.0;
    varr = 2.0 * gt3 / 3.0 - gt4 / 2.0 + 7.0 * gt5 / 30.0 - gt6 / 12.0 + 31.0 * gt7 / 1260.0 - gt8 / 160.0 +
           127.0 * gt9 / 90720.0;
    varv = 2.0 * gt - 2.0 * gt2 + 4.0 * gt3 / 3.0 - 2.0 * gt4 / 3.0 + 4.0 * gt5 / 15.0 - 4.0 * gt6 / 45.0 +
           8.0 * gt7 / 315.0 - 2.0 * gt8 / 315.0 + 4.0 * gt9 / 2835.0;
    crv = sqrt(3.0) * (0.5 - 3.0 * gt / 16.0 - 17.0 * gt2 / 1280.0 + 17.0 * gt3 / 6144.0 +
                       40967.0 * gt4 / 34406400.0 - 57203.0 * gt5 / 275251200.0 - 1429487.0 * gt6 / 13212057600.0);
  }
  if (step > 0)
    for (int i = 0; i < n; i++) {
      double tinvmass = t / mass[i];
      for (int c = 0; c < 3; c++) v[3 * i + c] += (1.0 - c0 / c1) * f[3 * i + c] * tinvmass / gammat;
    }
  double ekin = kinetic(n, v, mass);
  if (step < (steps - 1))
    for (int i = 0; i < n; i++) {
      double tinvmass = t / mass[i];
      double kTdivm = c_kB * temp / mass[i];
      double sigmav = sqrt(kTdivm * varv);
      double sigmar = sqrt(kTdivm * varr) / gamma;
      const double *nr = normals + 6 * i;
      double n1x = nr[0], n2y = nr[1], n2x = nr[2], n1z = nr[3], n1y = nr[4], n2z = nr[5];
      double dvv[3] = {sigmav * (crv * n1x + sqrt(1.0 - sqr(crv)) * n2x),
                       sigmav * (crv * n1y + sqrt(1.0 - sqr(crv)) * n2y),
                       sigmav * (crv * n1z + sqrt(1.0 - sqr(crv)) * n2z)};
      double drr[3] = {sigmar * n1x, sigmar * n1y, sigmar * n1z};
      for (int c = 0; c < 3; c++) {
        double dr = t * (c1 * v[3 * i + c] + c2 * f[3 * i + c] * tinvmass) + drr[c];
        dr *= 1 / c_Angstrom;
        double dv = (c0 * c2) * f[3 * i + c] * tinvmass / c1 + dvv[c];
        x[3 * i + c] += dr;
        v[3 * i + c] *= c0;
        v[3 * i + c] += dv;
      }
    }
  return ekin;
}

/* ------------------------------------------------------------------ LCPO */
#define LCPO_NMAX 80 /* lcpo.h: Nlistmax */

/* Maths::sphereSurfaceOverlap (maths/maths.cpp:103-106) */
static double lcpo_overlap(double ri, double rj, double dij) {
  return 2.0 * kPI * ri * (ri - dij / 2.0 - (ri * ri - rj * rj) / (2.0 * dij));
}

/* Distances as the reference's vector helpers form them: the free
 * function sqrdist(a, b) takes a - b, the member a.sqrdist(b) takes b - a
 * (maths/maths_vector.h:239-249, 352-368); the squares are the same. */
static double lcpo_sqrdist(const double *a, const double *b) {
  double g = a[0] - b[0], h = a[1] - b[1], j = a[2] - b[2];
  return g * g + h * h + j * j;
}

double pdo_lcpo(int n, const double *pos, const int *ptr, const int *data,
                const double *radius, const double *p, const double *sigma,
                const int8_t *use, int energy_only, double *sasa,
                double *deriv, long *truncated) {
  const double TwoPI = 2.0 * kPI, FourPI = 4.0 * kPI;
  int *cnt = calloc((size_t)n, sizeof(int));
  int *nl = malloc(sizeof(int) * (size_t)n * LCPO_NMAX);
  double *sv = malloc(sizeof(double) * (size_t)n * LCPO_NMAX);
  long lost = 0;
  /* overlap lists: pairs j < i of the neighbour list, i ascending, both
   * ends appended while they have room (lcpo.cpp:434-485, 688-746) */
  for (int i = 0; i < n; i++) {
    if (!use[i]) continue;
    const double *pi = pos + 3 * (size_t)i;
    const double ri = radius[i];
    for (int q = ptr[i]; q < ptr[i + 1]; q++) {
      int j = data[q] & 0x00FFFFFF;
      if (j >= i) break;
      if (!use[j]) continue;
      const double *pj = pos + 3 * (size_t)j;
      const double rj = radius[j];
      double sij, sji;
      if (energy_only) {
        double d = sqrt(lcpo_sqrdist(pi, pj));
        if (!(d < ri + rj)) continue;
        sij = lcpo_overlap(ri, rj, d);
        if (sij < 0) sij = 0;
        sji = lcpo_overlap(rj, ri, d);
        if (sji < 0) sji = 0;
      } else {
        double d2 = lcpo_sqrdist(pi, pj);
        if (!(d2 < (ri + rj) * (ri + rj))) continue;
        double d = sqrt(d2);
        double inv = 1 / d;
        double h = 0.5 * (ri * ri - rj * rj) * inv;
        sij = TwoPI * ri * (ri - d * 0.5 - h);
        sji = TwoPI * rj * (rj - d * 0.5 + h);
      }
      if (cnt[i] < LCPO_NMAX) {
        nl[(size_t)i * LCPO_NMAX + cnt[i]] = j;
        sv[(size_t)i * LCPO_NMAX + cnt[i]] = sij;
        cnt[i]++;
      } else {
        lost++;
      }
      if (cnt[j] < LCPO_NMAX) {
        nl[(size_t)j * LCPO_NMAX + cnt[j]] = i;
        sv[(size_t)j * LCPO_NMAX + cnt[j]] = sji;
        cnt[j]++;
      } else {
        lost++;
      }
    }
  }
  double epot = 0;
  for (int i = 0; i < n; i++) {
    double *di = deriv ? deriv + 3 * (size_t)i : NULL;
    if (!energy_only) di[0] = di[1] = di[2] = 0;
    if (!use[i]) {
      sasa[i] = 0;
      continue;
    }
    const double *pi = pos + 3 * (size_t)i;
    const double ri = radius[i];
    const double Si = FourPI * ri * ri; /* sphereSurfaceArea, maths.cpp:97-100 */
    double Si2 = 0, Si3 = 0, Si4 = 0;
    double a2[3] = {0, 0, 0}, a4[3] = {0, 0, 0};
    for (int e = 0; e < cnt[i]; e++) {
      const int ja = nl[(size_t)i * LCPO_NMAX + e];
      const double *pj = pos + 3 * (size_t)ja;
      const double Si2_t = sv[(size_t)i * LCPO_NMAX + e];
      double Si3_t = 0;
      if (energy_only) {
        /* lcpo.cpp:517-537 */
        for (int k = 0; k < cnt[ja]; k++) {
          const int ka = nl[(size_t)ja * LCPO_NMAX + k];
          if (ka == i) continue;
          if (ri + radius[ka] < sqrt(lcpo_sqrdist(pos + 3 * (size_t)ka, pi))) continue;
          Si3_t += sv[(size_t)ja * LCPO_NMAX + k];
        }
      } else {
        /* lcpo.cpp:772-901 */
        const double rj = radius[ja];
        double Si3ik_t = 0;
        const double dij = sqrt(lcpo_sqrdist(pj, pi));
        const double invij = 1 / dij;
        double h = 0.5 * (ri * ri - rj * rj) * invij;
        const double sji = TwoPI * rj * (rj - dij * 0.5 + h);
        h *= 2.0 * invij;
        double d2[3], d3[3] = {0, 0, 0}, d4[3], d3b[3] = {0, 0, 0}, d4b[3] = {0, 0, 0}, a2t[3], ddd[3];
        double dAdd = kPI * rj * (-h - 1);
        for (int c = 0; c < 3; c++) ddd[c] = -(pi[c] - pj[c]) / dij;
        for (int c = 0; c < 3; c++) d2[c] = dAdd * ddd[c];
        dAdd = kPI * ri * (h - 1);
        for (int c = 0; c < 3; c++) a2t[c] = dAdd * ddd[c];
        for (int k = 0; k < cnt[ja]; k++) {
          const int ka = nl[(size_t)ja * LCPO_NMAX + k];
          const double *pk = pos + 3 * (size_t)ka;
          const double rk = radius[ka];
          if (ka == i) continue;
          double dik = lcpo_sqrdist(pk, pi);
          if ((ri + rk) * (ri + rk) < dik) continue;
          dik = sqrt(dik);
          const double invik = 1 / dik;
          const double hk = (ri * ri - rk * rk) * (invik * invik);
          dAdd = kPI * ri * (hk - 1);
          double dk[3];
          for (int c = 0; c < 3; c++) dk[c] = -(pi[c] - pk[c]) * invik;
          const double sjk = sv[(size_t)ja * LCPO_NMAX + k];
          for (int c = 0; c < 3; c++) d3[c] += dAdd * dk[c];
          dAdd = kPI * rk * (-hk - 1);
          Si3ik_t += kPI * ri * (2 * ri - dik - dik * hk);
          for (int c = 0; c < 3; c++) d3b[c] += dAdd * dk[c];
          for (int c = 0; c < 3; c++) d4b[c] += sjk * dAdd * dk[c];
          Si3_t += sjk;
        }
        for (int c = 0; c < 3; c++) d4[c] = sji * d3[c] + d4b[c];
        for (int c = 0; c < 3; c++) d3[c] += d3b[c];
        for (int c = 0; c < 3; c++) d4[c] += d2[c] * Si3ik_t;
        const double *pj4 = p + 4 * (size_t)ja;
        const double m2 = pj4[1] * sigma[ja], m3 = pj4[2] * sigma[ja], m4 = pj4[3] * sigma[ja];
        for (int c = 0; c < 3; c++) {
          d2[c] *= m2;
          d3[c] *= m3;
          d4[c] *= m4;
        }
        for (int c = 0; c < 3; c++) di[c] += d2[c];
        for (int c = 0; c < 3; c++) di[c] += d3[c];
        for (int c = 0; c < 3; c++) di[c] += d4[c];
        for (int c = 0; c < 3; c++) a2[c] += a2t[c];
        for (int c = 0; c < 3; c++) a4[c] += Si3_t * a2t[c];
      }
      Si4 += Si3_t * Si2_t;
      Si3 += Si3_t;
      Si2 += Si2_t;
    }
    const double *pi4 = p + 4 * (size_t)i;
    double SAi = pi4[0] * Si + pi4[1] * Si2 + pi4[2] * Si3 + pi4[3] * Si4;
    if (!energy_only) {
      const double m2 = pi4[1] * sigma[i], m4 = pi4[3] * sigma[i];
      for (int c = 0; c < 3; c++) {
        a2[c] *= m2;
        a4[c] *= m4;
      }
      for (int c = 0; c < 3; c++) di[c] += a2[c];
      for (int c = 0; c < 3; c++) di[c] += a4[c];
    }
    if (SAi < 0) {
      SAi = 0;
      if (!energy_only) di[0] = di[1] = di[2] = 0;
    }
    sasa[i] = SAi;
    epot += SAi * sigma[i];
  }
  free(cnt);
  free(nl);
  free(sv);
  if (truncated) *truncated = lost;
  return epot;
}
