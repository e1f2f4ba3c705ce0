// FF_Bonded on the device: harmonic bonds (ffbonded.cpp:885-940), harmonic
// angles (:994-1129) and Fourier / harmonic dihedrals for torsions and
// impropers (calcDihedralForces, :1207-1499).  One thread per term, FP64
// arithmetic (the terms are O(N) and cheap), forces scattered with 64-bit
// fixed-point atomics (order-independent), per-term energies reduced per
// system in a fixed order.
#include <cuda_runtime.h>

#include "internal.cuh"

namespace pdgpu {

__device__ __forceinline__ void add_force(const PackView &v, int i, double fx, double fy, double fz) {
  atomicAdd((unsigned long long *)&v.fx[i], (unsigned long long)__double2ll_rn(fx * kForceScale));
  atomicAdd((unsigned long long *)&v.fy[i], (unsigned long long)__double2ll_rn(fy * kForceScale));
  atomicAdd((unsigned long long *)&v.fz[i], (unsigned long long)__double2ll_rn(fz * kForceScale));
}

__device__ __forceinline__ void bond_term(const PackView &v, int t, double *e_term, double *vir_term) {
  int2 ij = v.bt.bij[t];
  double2 lk = v.bt.blk[t];
  int i = ij.x, j = ij.y;
  double bx = v.x[i] - v.x[j], by = v.y[i] - v.y[j], bz = v.z[i] - v.z[j];
  double d2 = bx * bx + by * by + bz * bz;
  double inv_d = rsqrt(d2);
  double d = d2 * inv_d;
  double fm = 2 * lk.y * (d - lk.x);
  e_term[t] = lk.y * (d - lk.x) * (d - lk.x);
  vir_term[t] = d * fm;
  double s = fm * inv_d;
  add_force(v, i, -bx * s, -by * s, -bz * s);
  add_force(v, j, bx * s, by * s, bz * s);
}

__device__ __forceinline__ void angle_term(const PackView &v, int t, double *e_term) {
  double2 kt = v.bt.akt[t];
  e_term[t] = 0.0;
  if (kt.x == 0) return;
  int4 q = v.bt.aiaj[t];
  int i = q.x, a = q.y, j = q.z;
  double iv[3] = {v.x[i] - v.x[a], v.y[i] - v.y[a], v.z[i] - v.z[a]};
  double jv[3] = {v.x[j] - v.x[a], v.y[j] - v.y[a], v.z[j] - v.z[a]};
  double inv_iv = rsqrt(iv[0] * iv[0] + iv[1] * iv[1] + iv[2] * iv[2]);
  double inv_jv = rsqrt(jv[0] * jv[0] + jv[1] * jv[1] + jv[2] * jv[2]);
  double ui[3], uj[3];
  for (int c = 0; c < 3; c++) {
    ui[c] = iv[c] * inv_iv;
    uj[c] = jv[c] * inv_jv;
  }
  double cs = ui[0] * uj[0] + ui[1] * uj[1] + ui[2] * uj[2];
  double theta = acos(cs);
  double sn = sqrt(fmax(0.0, 1.0 - cs * cs));  // sin(acos(cs)) without a second transcendental
  double dth = theta - kt.y;
  e_term[t] = kt.x * dth * dth;
  double fm = 2 * kt.x * dth;
  double bi[3], bj[3];
  const double gi = fm * inv_iv / sn, gj = fm * inv_jv / sn;
  for (int c = 0; c < 3; c++) {
    bi[c] = gi * (ui[c] * cs - uj[c]);
    bj[c] = gj * (uj[c] * cs - ui[c]);
  }
  add_force(v, i, -bi[0], -bi[1], -bi[2]);
  add_force(v, j, -bj[0], -bj[1], -bj[2]);
  add_force(v, a, bi[0] + bj[0], bi[1] + bj[1], bi[2] + bj[2]);
}

__device__ __forceinline__ void dihedral_term(const PackView &v, int t, double *e_term) {
  int4 q = v.bt.tidx[t];
  int ti = q.x, ta = q.y, tb = q.z, tj = q.w;
  const int ty = v.bt.ttype[t];
  const double *par = v.bt.tpar + 20 * (size_t)ty;
  int terms = v.bt.tterms[ty];
  double a[3] = {v.x[ti] - v.x[ta], v.y[ti] - v.y[ta], v.z[ti] - v.z[ta]};
  double b[3] = {v.x[ta] - v.x[tb], v.y[ta] - v.y[tb], v.z[ta] - v.z[tb]};
  double c[3] = {v.x[tb] - v.x[tj], v.y[tb] - v.y[tj], v.z[tb] - v.z[tj]};
  double n1[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  double n2[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
  double n3[3] = {b[1] * n1[2] - b[2] * n1[1], b[2] * n1[0] - b[0] * n1[2], b[0] * n1[1] - b[1] * n1[0]};
  double in1 = rsqrt(n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]);
  double in2 = rsqrt(n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
  double in3 = rsqrt(n3[0] * n3[0] + n3[1] * n3[1] + n3[2] * n3[2]);
  double cos_phi = (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]) * in1 * in2;
  double sin_phi = (n3[0] * n2[0] + n3[1] * n2[1] + n3[2] * n2[2]) * in3 * in2;
  for (int k = 0; k < 3; k++) n2[k] *= in2;
  // phi = -atan2(sin_phi, cos_phi) (ffbonded.cpp:1261); the Fourier terms
  // with integer periodicity 1..6 need only cos(n phi) and sin(n phi), from
  // powers of cos(phi) + i sin(phi); phi itself only for the others
  const double hinv = rsqrt(cos_phi * cos_phi + sin_phi * sin_phi);
  const double c1 = cos_phi * hinv, s1 = -sin_phi * hinv;
  bool need_phi = false;
  for (int m = 0; m < terms; m++) {
    double n = par[4 + m];
    need_phi |= !(n > 0 && n <= 6 && n == floor(n));
  }
  double phi = need_phi ? -atan2(sin_phi, cos_phi) : 0.0;
  bool use_cos = fabs(sin_phi) > 0.1;
  double d1[3], d2[3];
  if (use_cos) {
    for (int k = 0; k < 3; k++) n1[k] *= in1;
    for (int k = 0; k < 3; k++) {
      d1[k] = in1 * (n1[k] * cos_phi - n2[k]);
      d2[k] = in2 * (n2[k] * cos_phi - n1[k]);
    }
  } else {
    for (int k = 0; k < 3; k++) n3[k] *= in3;
    for (int k = 0; k < 3; k++) {
      d1[k] = in3 * (n3[k] * sin_phi - n2[k]);  // dsin/dn3
      d2[k] = in2 * (n2[k] * sin_phi - n3[k]);  // dsin/dn2
    }
  }
  // the force is linear in dE/dphi: sum it over the Fourier terms, then
  // apply the geometry once
  double e = 0, dEs = 0;
  const double PI = 3.14159265358979323846;
  for (int m = 0; m < terms; m++) {
    double k = par[m], n = par[4 + m], gamma = par[8 + m];
    double ep, dE;
    if (n > 0 && n <= 6 && n == floor(n)) {
      // cos(n phi + gamma), sin(n phi + gamma) from (c1 + i s1)^n
      double cn = c1, sn = s1;
      for (int p = 1; p < (int)n; p++) {
        double t = cn * c1 - sn * s1;
        sn = sn * c1 + cn * s1;
        cn = t;
      }
      const double cg = par[12 + m], sg = par[16 + m];
      double cv = cn * cg - sn * sg, sv = sn * cg + cn * sg;
      ep = k * (1.0 + cv);
      dE = -n * k * sv;
    } else if (n > 0) {
      double sv, cv;
      sincos(n * phi + gamma, &sv, &cv);
      ep = k * (1.0 + cv);
      dE = -n * k * sv;
    } else {
      double diff = phi - gamma;
      if (diff < -PI)
        diff += 2.0 * PI;
      else if (diff > PI)
        diff -= 2.0 * PI;
      ep = k * diff * diff;
      dE = 2.0 * k * diff;
    }
    e += ep;
    dEs += dE;
  }
  double fi[3], fab[3], fj[3];
  if (use_cos) {
    const double dE = dEs / sin_phi;
    fi[0] = dE * (b[1] * d1[2] - b[2] * d1[1]);
    fi[1] = dE * (b[2] * d1[0] - b[0] * d1[2]);
    fi[2] = dE * (b[0] * d1[1] - b[1] * d1[0]);
    fj[0] = dE * (b[2] * d2[1] - b[1] * d2[2]);
    fj[1] = dE * (b[0] * d2[2] - b[2] * d2[0]);
    fj[2] = dE * (b[1] * d2[0] - b[0] * d2[1]);
    fab[0] = dE * (a[2] * d1[1] - a[1] * d1[2] + c[1] * d2[2] - c[2] * d2[1]);
    fab[1] = dE * (a[0] * d1[2] - a[2] * d1[0] + c[2] * d2[0] - c[0] * d2[2]);
    fab[2] = dE * (a[1] * d1[0] - a[0] * d1[1] + c[0] * d2[1] - c[1] * d2[0]);
  } else {
    const double dE = dEs / -cos_phi;
    fi[0] = dE * ((b[1] * b[1] + b[2] * b[2]) * d1[0] - b[0] * b[1] * d1[1] - b[0] * b[2] * d1[2]);
    fi[1] = dE * ((b[2] * b[2] + b[0] * b[0]) * d1[1] - b[1] * b[2] * d1[2] - b[1] * b[0] * d1[0]);
    fi[2] = dE * ((b[0] * b[0] + b[1] * b[1]) * d1[2] - b[2] * b[0] * d1[0] - b[2] * b[1] * d1[1]);
    fj[0] = dE * (d2[1] * b[2] - d2[2] * b[1]);
    fj[1] = dE * (d2[2] * b[0] - d2[0] * b[2]);
    fj[2] = dE * (d2[0] * b[1] - d2[1] * b[0]);
    fab[0] = dE * (-(b[1] * a[1] + b[2] * a[2]) * d1[0] + (2.0 * b[0] * a[1] - a[0] * b[1]) * d1[1] +
                   (2.0 * b[0] * a[2] - a[0] * b[2]) * d1[2] + d2[2] * c[1] - d2[1] * c[2]);
    fab[1] = dE * (-(b[2] * a[2] + b[0] * a[0]) * d1[1] + (2.0 * b[1] * a[2] - a[1] * b[2]) * d1[2] +
                   (2.0 * b[1] * a[0] - a[1] * b[0]) * d1[0] + d2[0] * c[2] - d2[2] * c[0]);
    fab[2] = dE * (-(b[0] * a[0] + b[1] * a[1]) * d1[2] + (2.0 * b[2] * a[0] - a[2] * b[0]) * d1[0] +
                   (2.0 * b[2] * a[1] - a[2] * b[1]) * d1[1] + d2[1] * c[0] - d2[0] * c[1]);
  }
  e_term[t] = e;
  add_force(v, ti, fi[0], fi[1], fi[2]);
  add_force(v, ta, fab[0] - fi[0], fab[1] - fi[1], fab[2] - fi[2]);
  add_force(v, tb, fj[0] - fab[0], fj[1] - fab[1], fj[2] - fab[2]);
  add_force(v, tj, -fj[0], -fj[1], -fj[2]);
}

// One launch for every bonded term: threads [0, nb) bonds, then angles,
// then torsions and impropers.  Per-term energies feed the energy reduction.
__global__ void k_bonded_all(PackView v) {
  PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;  // the step is being re-planned
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const BondedTerms &b = v.bt;
  if (t < b.nb) {
    bond_term(v, t, b.e_bond, b.vir_bond);
    return;
  }
  t -= b.nb;
  if (t < b.na) {
    angle_term(v, t, b.e_angle);
    return;
  }
  t -= b.na;
  if (t < b.nt + b.ni) dihedral_term(v, t, b.e_dih);
}

void launch_bonded_terms(const PackView &v, cudaStream_t st) {
  const BondedTerms &b = v.bt;
  int n = b.nb + b.na + b.nt + b.ni;
  if (n) PDGPU_LAUNCH_DEP(k_bonded_all, (n + 127) / 128, 128, 0, st, v);
}

}  // namespace pdgpu
