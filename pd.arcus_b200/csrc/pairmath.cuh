// Per-pair arithmetic shared by the row kernels (pair.cu) and the
// cluster-pair tile kernels (tiles.cu), so that both evaluate every
// interaction with the same instructions.
#pragma once
#include "internal.cuh"

namespace pdgpu {

template <int W, typename T>
__device__ __forceinline__ T group_sum(T x) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// The reference's squared distance with its operand order and no
// contraction: sqrdist(v1,v2) = (g*g + h*h) + j*j, g = v1.x - v2.x
// (neighbourlist.cpp:263-264, gbff.cpp:1553-1556, maths_vector.h:104-107).
// IEEE subtraction is antisymmetric, so either argument order gives the
// same value.
__device__ __forceinline__ double ref_d2(double ax, double ay, double az, double bx, double by, double bz) {
  double g = __dsub_rn(ax, bx), h = __dsub_rn(ay, by), k = __dsub_rn(az, bz);
  return __dadd_rn(__dadd_rn(__dmul_rn(g, g), __dmul_rn(h, h)), __dmul_rn(k, k));
}

// hi + lo coordinate difference of records a (hi) / b (lo): p_i - p_j.
// The square is spelled out with explicit FMAs so every kernel (row or
// tile, i or j side) gets the same bits for a pair: d(j,i) = -d(i,j)
// exactly, and the square does not depend on how a compiler contracts.
struct Dx {
  float x, y, z, r2;
};
__device__ __forceinline__ Dx diff(const float4 &ia, const float4 &ib, const float4 &ja, const float4 &jb) {
  Dx d;
  d.x = __fadd_rn(__fsub_rn(ia.x, ja.x), __fsub_rn(ib.x, jb.x));
  d.y = __fadd_rn(__fsub_rn(ia.y, ja.y), __fsub_rn(ib.y, jb.y));
  d.z = __fadd_rn(__fsub_rn(ia.z, ja.z), __fsub_rn(ib.z, jb.z));
  d.r2 = __fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, __fmul_rn(d.x, d.x)));
  return d;
}

// BondOrder as the neighbour list encodes it (neighbourlist.cpp:279-290,
// bondorder.cpp:170-195): the band for |i-j| < MaxIndexDelta, else the
// off-diagonal corrections (neighbourlist.cpp:162-203), else 7.
__device__ __forceinline__ int bond_order(const PackView &v, int s, int i, int j) {
  int o = v.atom_off[s];
  int li = i - o, lj = j - o;
  int delta = li > lj ? li - lj : lj - li;
  int mid = v.mid[s];
  if (delta < mid) {
    int lo = li < lj ? li : lj;
    return v.band[v.band_off[s] + (long long)lo * mid + (delta - 1)];
  }
  int b = v.off_ptr[i], e = v.off_ptr[i + 1];
  for (int k = b; k < e; k++)
    if (v.off_data[k].x == j) return v.off_data[k].y & 7;
  return 7;
}

// Exact FP64 re-evaluation of the reference's GB branch predicate
// uGB = -srij*0.25/aiaj > ExpApproxThreshold, with srij formed as in
// gbff.cpp:1553-1556 (dddx = p_i - p_j; sqr+sqr+sqr).
// (Plain pointer arguments: taking the address of a kernel's PackView
// parameter would copy it to local memory in every thread.)
__device__ __forceinline__ bool gb_branch_exact(const double *__restrict__ x, const double *__restrict__ y,
                                                const double *__restrict__ z, const double *__restrict__ born,
                                                int i, int j, double thr) {
  double srij = ref_d2(x[i], y[i], z[i], x[j], y[j], z[j]);
  double aiaj = born[i] * born[j];
  double uGB = -srij * 0.25 / aiaj;
  return uGB > thr;
}

// Settings of the fused GB + LJ + Coulomb pass, in registers.
struct GbSettings {
  float thr, band, rc2, rin, inv_sw2, elec14, vdw14, econv_in, econv_out, premul, vdw_rc, vdw_rin, vdw_inv_sw2;
  double thr_d;
  // FastMode off (calcBornForces, gbff.cpp:1172-1330): no vacuum LJ/Coulomb
  // in this pass (FF_NonBonded::calcForces gives them), and beyond the
  // exp-approximation range the GB term keeps its t = 0 limit q_i q_j / r
  bool slow;
  __device__ __forceinline__ void load(const SysParams &P) {
    slow = P.fast_mode == 0;
    thr = P.exp_thresh;
    thr_d = P.exp_thresh_d;
    band = 4e-6f * fabsf(thr);
    rc2 = P.rc2;
    rin = P.rin;
    inv_sw2 = P.inv_sw2;
    elec14 = P.elec14;
    vdw14 = P.vdw14;
    econv_in = P.econv_in;
    econv_out = P.econv_out;
    premul = P.premul;
    vdw_rc = P.vdw_rc;
    vdw_rin = P.vdw_rin;
    vdw_inv_sw2 = P.vdw_inv_sw2;
  }
};

// One interaction of calcForcesIncludingVacuo loop 1 (gbff.cpp:1542-1719)
// for a pair already known to lie within Rc: the radial force factor
// (force on i = -fscal * (p_i - p_j)), the GB pair energy, dE/da (per unit
// of the partner's radius), the LJ and Coulomb energies.  All selections
// are branch-free except the LJ block (skipped for 1-2/1-3 partners and
// beyond the VdW cutoff) and the rare FP64 re-decision of the GB branch.
struct GbPair {
  float fscal, epol, dedal, vdw, elec;
};
__device__ __forceinline__ GbPair gb_pair_term(const GbSettings &g, const Dx &d, bool nb, bool b14, float ai,
                                               float aj, float qi, float qj, float radi, float radj, float epsi,
                                               float epsj, const PackView &v, int i, int j) {
  GbPair o;
  const float invr = rsqrtf(d.r2);
  const float r = d.r2 * invr;
  const float qiqj = qi * qj;
  const float aiaj = ai * aj;
  const float u = __fdividef(-0.25f * d.r2, aiaj);
  bool gb = u > g.thr;
  if (fabsf(u - g.thr) <= g.band) gb = gb_branch_exact(v.x, v.y, v.z, v.born_d, i, j, g.thr_d);
  // energy switch (applies to GB and Coulomb, gbff.cpp:1602-1614)
  const float dr = r - g.rin;
  const float sw = 1.f - g.inv_sw2 * dr * dr;
  const bool on = r >= g.rin;
  const float S = on ? sw * sw : 1.f;
  const float dSdd = on ? -4.f * g.inv_sw2 * dr * sw : 0.f;
  // GB cross term (all bond orders) where the exp approximation applies
  // (a branch: partners beyond about 4 sqrt(a_i a_j) skip it together)
  float dedr = 0.f;
  o.epol = 0.f;
  o.dedal = 0.f;
  if (gb) {
    const float tg = __expf(u);
    const float fgb = rsqrtf(d.r2 + tg * aiaj);
    const float l = fgb * fgb;
    const float epol0 = g.premul * qiqj * fgb;
    const float dedr0 = -epol0 * (r - 0.25f * r * tg) * l;
    const float dedal0 = -epol0 * tg * (1.f - u) * l;
    o.epol = epol0 * S;
    dedr = S * dedr0 + dSdd * epol0;
    o.dedal = dedal0 * S;
  } else if (g.slow) {
    const float epol0 = g.premul * qiqj * invr;
    o.epol = epol0 * S;
    dedr = S * (-epol0 * invr) + dSdd * epol0;
  }
  if (g.slow) nb = false;  // the vacuum terms come from FF_NonBonded::calcForces
  // vacuum Coulomb at the solute (GB branch) or solvent dielectric
  const float ec = nb ? (gb ? g.econv_in : g.econv_out) * (b14 ? g.elec14 : 1.f) * qiqj * invr : 0.f;
  const float elf = S * (-ec * invr) + ec * dSdd;
  o.elec = ec * S;
  // Lennard-Jones 12-6 with its own switch
  float vdw = 0.f, vdwf = 0.f;
  if (nb && r < g.vdw_rc) {
    const float rr = (radi + radj) * invr;
    const float rr2 = rr * rr;
    const float B = rr2 * rr2 * rr2;
    const float A = B * B;
    const float eps = epsi * epsj * (b14 ? g.vdw14 : 1.0f);
    vdw = (2.f * eps) * (0.5f * A - B);
    vdwf = -(12.f * eps * invr) * (A - B);
    const float vd = r - g.vdw_rin;
    const float vs = 1.f - g.vdw_inv_sw2 * vd * vd;
    const bool von = r > g.vdw_rin;
    const float vS = von ? vs * vs : 1.f;
    const float vdS = von ? -4.f * g.vdw_inv_sw2 * vd * vs : 0.f;
    vdwf = vS * vdwf + vdw * vdS;
    vdw *= vS;
  }
  o.vdw = vdw;
  o.fscal = dedr * 2.f * invr + (vdwf + elf) * invr;
  return o;
}

// One term of the Born-radius chain rule (gbff.cpp:1758-1806) for a pair
// within the Still cutoff: the radial factor tt, force on i = tt*(p_i-p_j).
// Symmetric in i and j.
__device__ __forceinline__ float chain_term(const Dx &d, float Ri, float Rj, float Vi, float Vj, float wi,
                                            float wj, float invP5, float piP5, float P4) {
  const float Rs = Ri + Rj;
  const float rdivR = __fdividef(d.r2, Rs * Rs);
  float X = 4.f;
  if (!(rdivR > invP5)) {
    const float th = rdivR * piP5;
    float sn, cs;
    __sincosf(th, &sn, &cs);
    const float sq = 0.5f - 0.5f * cs;
    X = 4.f * sq * sq - 2.f * sq * sn * th;
  }
  const float ir2 = __fdividef(1.f, d.r2);  // the fast reciprocal: deterministic, ~1 ulp
  const float ir6 = ir2 * ir2 * ir2;
  return P4 * X * ir6 * (wi * Vj + wj * Vi);
}

// One Born-sum term P4*V/r^4 * CCF (gbff.cpp:440-462) for a pair within the
// Still cutoff, scaled by `scale` (the fixed-point unit) and without V:
// the caller multiplies by the partner's V.  CCF is symmetric in i and j.
__device__ __forceinline__ float born_term_noV(const Dx &d, float Ri, float Rj, float invP5, float piP5,
                                               float P4scaled) {
  // explicit roundings: the i and j sides of a pair, in any kernel, get
  // the same bits
  const float Rs = __fadd_rn(Ri, Rj);
  const float ir2 = __fdividef(1.f, d.r2);  // the fast reciprocal: deterministic, ~1 ulp
  float term = __fmul_rn(__fmul_rn(P4scaled, ir2), ir2);
  const float rdivR = __fdividef(d.r2, __fmul_rn(Rs, Rs));
  if (!(rdivR > invP5)) {
    // CCF = (1/2 - 1/2 cos(pi P5 r^2/(Ri+Rj)^2))^2 = sin^4(pi P5 r^2/(2 (Ri+Rj)^2))
    const float sh = __sinf(__fmul_rn(__fmul_rn(0.5f, piP5), rdivR));
    const float c = __fmul_rn(sh, sh);
    term = __fmul_rn(term, __fmul_rn(c, c));
  }
  return term;
}

}  // namespace pdgpu
