// Pair kernels of the Still GB + LJ + Coulomb evaluation.
//
//   K2 k_born        calcBornRadii_PairwiseApprox     (gbff.cpp:415-466)
//   K3 k_gb_pair     calcForcesIncludingVacuo loop 1  (gbff.cpp:1529-1736)
//   K4 k_gb_chain    calcForcesIncludingVacuo loop 2  (gbff.cpp:1751-1818)
//      k_born_energy calcBornEnergy                   (gbff.cpp:520-579)
//      k_nonbonded   FF_NonBonded_CalcForces_T_fast2  (nonbonded.cpp:548-893)
//
// Layout: one warp per atom i walks i's full neighbour row (lanes stride the
// row; rows are contiguous uint32 (j<<3|bondorder) entries).  Every atom
// accumulates only its own force, so no atomics touch j; per-lane partials
// are converted to 64-bit fixed point and summed with shuffles, so every
// result is bit-reproducible run to run and independent of lane order.
//
// Precision: pair arithmetic in FP32 on coordinates split as hi+lo floats
// (dx = (xi_hi - xj_hi) + (xi_lo - xj_lo), i.e. the FP64 difference rounded
// once).  The two discontinuous predicates of the reference -- the Still
// cutoff (Born sums, chain rule) and the GB exp-approximation threshold
// (uGB > -4 switches the solvent term off and Coulomb to eps=80) -- are
// decided in FP64 with the reference's exact expressions whenever the FP32
// value lies within a guard band of the threshold.  Born sums are FP64 per
// term (they feed the threshold through a_i*a_j) and fixed point across
// lanes; energies are FP64 sums of per-lane FP32 partials.
//
// Roofline: FP32/SFU-bound.  Algorithmic work per interaction: K2 21 flop +
// 3 SFU (directed pairs r<=10A, bo>=3), K3 90 flop + 5 SFU (unordered pairs
// r<=Rc), K4 36 flop + 4 SFU (as K2).
#include <cuda_runtime.h>

#include "internal.cuh"

namespace pdgpu {

__device__ __forceinline__ long long warp_sum_ll(long long x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ long long to_fixed_force(float f) {
  // kcal/mol/A -> 2^32 fixed point; saturate far outside any physical range
  float s = f * (float)kForceScale;
  s = fminf(fmaxf(s, -9.0e18f), 9.0e18f);
  return __float2ll_rn(s);
}

// Reciprocal of a double by one FP32 seed and two Newton-Raphson steps
// (quadratic convergence: 2^-23 -> 2^-46 -> below double rounding).
__device__ __forceinline__ double rcp_d(double a) {
  double y = (double)__frcp_rn(__double2float_rn(a));
  double e = fma(-a, y, 1.0);
  y = fma(y, e, y);
  e = fma(-a, y, 1.0);
  return fma(y, e, y);
}

// The reference's squared distance with its operand order and no
// contraction: sqrdist(v1,v2) = (g*g + h*h) + j*j, g = v1.x - v2.x.
__device__ __forceinline__ double ref_d2(double ax, double ay, double az, double bx, double by,
                                         double bz) {
  double g = __dsub_rn(ax, bx), h = __dsub_rn(ay, by), k = __dsub_rn(az, bz);
  return __dadd_rn(__dadd_rn(__dmul_rn(g, g), __dmul_rn(h, h)), __dmul_rn(k, k));
}

// --------------------------------------------------------------- positions
// FP64 state -> (hi, lo) float copies used by the pair kernels.
__global__ void k_pack_positions(PackView v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  double x = v.x[i], y = v.y[i], z = v.z[i];
  float hx = __double2float_rn(x), hy = __double2float_rn(y), hz = __double2float_rn(z);
  float4 a = v.pa[i];
  a.x = hx;
  a.y = hy;
  a.z = hz;
  v.pa[i] = a;
  v.pb[i] = make_float4(__double2float_rn(x - (double)hx), __double2float_rn(y - (double)hy),
                        __double2float_rn(z - (double)hz), 0.f);
}

void launch_pack_positions(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_pack_positions, (v.n_atoms + 255) / 256, 256, 0, st, v);
}

__global__ void k_zero(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < v.n_atoms) {
    v.fx[i] = 0;
    v.fy[i] = 0;
    v.fz[i] = 0;
#pragma unroll
    for (int k = 0; k < AE_COUNT; k++) v.e_atom[(size_t)k * v.n_atoms + i] = 0.0;
  }
  if (i < v.n_sys * E_COUNT) {
    // keep the kinetic slots; zero the potential record (WorkSpace::zeroForces)
    int slot = i % E_COUNT;
    if (slot != E_EKIN) v.ene[i] = 0.0;
  }
}

void launch_zero(const PackView &v, cudaStream_t st) {
  int n = max(v.n_atoms, v.n_sys * E_COUNT);
  if (n) PDGPU_LAUNCH(k_zero, (n + 255) / 256, 256, 0, st, v);
}

// --------------------------------------------------------------- K2 radii
__global__ void __launch_bounds__(256) k_born(PackView v, int zero_first) {
  if (v.flags[F_NL_OVERFLOW]) return;  // list incomplete: the host re-plans
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const int s = v.sys_of[i];
  const SysParams &P = v.sp[s];
  if (zero_first && lane < 3) {
    // WorkSpace::zeroForces for this atom (and the record, by the first atom)
    long long *f = lane == 0 ? v.fx : (lane == 1 ? v.fy : v.fz);
    f[i] = 0;
    if (i == v.atom_off[s])
      for (int k = lane; k < E_COUNT; k += 3)
        if (k != E_EKIN) v.ene[(size_t)s * E_COUNT + k] = 0.0;
  }
  const double xi = v.x[i], yi = v.y[i], zi = v.z[i];
  const double Ri = v.gbR_d[i];
  const double still2 = P.still2_d;
  const double invP5 = P.invP5_d;
  const double P5 = P.P5_d;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  double acc = 0.0;
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    if ((ent & 7u) <= 2u) continue;  // 1-2 and 1-3 partners carry no Born term
    int j = (int)(ent >> 3);
    double d2 = ref_d2(xi, yi, zi, v.x[j], v.y[j], v.z[j]);
    if (d2 > still2) continue;
    double Rs = Ri + v.gbR_d[j];
    double s2 = Rs * Rs;
    double inv = rcp_d(d2);
    double term = v.pv_d[j] * inv * inv;
    if (!(d2 > s2 * invP5)) {
      // close-contact switching factor CCF (rare; exact division + FP64 cos)
      double rdivR = d2 / s2;
      double c = 0.5 - 0.5 * cos(rdivR * P5 * 3.14159265358979323846);
      if (!(rdivR > invP5)) term *= c * c;
    }
    acc += term;
  }
  long long fixed = warp_sum_ll(__double2ll_rn(acc * kBornScale));
  if (lane == 0) {
    double Gpol = v.terms123[i] + (double)fixed * kInvBornScale;
    double a = -P.halfeconv_d / Gpol + P.born_offset_d;
    v.born_d[i] = a;
    reinterpret_cast<float2 *>(v.born_f)[i] = make_float2((float)a, (float)(1.0 / a));
  }
}

void launch_born_radii(const PackView &v, cudaStream_t st, bool zero_first) {
  if (v.n_atoms) PDGPU_LAUNCH(k_born, (v.n_atoms + 7) / 8, 256, 0, st, v, (int)zero_first);
}

// --------------------------------------------------------------- K3 pair
// Exact FP64 re-evaluation of the reference's GB branch predicate
// uGB = -srij*0.25/aiaj > ExpApproxThreshold, with srij formed as in
// gbff.cpp:1553-1556 (dddx = p_i - p_j; sqr+sqr+sqr).
// (Plain pointer arguments: taking the address of the kernel's PackView
// parameter would copy it to local memory in every thread.)
__device__ __noinline__ bool gb_branch_exact(const double *__restrict__ x, const double *__restrict__ y,
                                             const double *__restrict__ z, const double *__restrict__ born,
                                             int i, int j, double thr) {
  double srij = ref_d2(x[i], y[i], z[i], x[j], y[j], z[j]);
  double aiaj = born[i] * born[j];
  double uGB = -srij * 0.25 / aiaj;
  return uGB > thr;
}

__global__ void __launch_bounds__(256) k_gb_pair(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pa[i], ib = v.pb[i], ip = v.prm[i];
  const float2 ab = reinterpret_cast<const float2 *>(v.born_f)[i];
  const float ai = ab.x, inv_ai = ab.y;
  const float qi = ia.w, radi = ip.x, epsi = ip.y;
  const float thr = P.exp_thresh;
  const float band = 4e-6f * fabsf(thr);
  float fx = 0.f, fy = 0.f, fz = 0.f;  // -dE/dr_i, kcal/mol/A
  float e_vdw = 0.f, e_el = 0.f, e_pol = 0.f, deda = 0.f;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int j = (int)(ent >> 3);
    int bo = (int)(ent & 7u);
    float4 ja = v.pa[j], jb = v.pb[j];
    float dx = (ia.x - ja.x) + (ib.x - jb.x);
    float dy = (ia.y - ja.y) + (ib.y - jb.y);
    float dz = (ia.z - ja.z) + (ib.z - jb.z);
    float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > P.rc2) continue;
    float invr = rsqrtf(r2);
    float r = r2 * invr;
    float2 jbf = reinterpret_cast<const float2 *>(v.born_f)[j];
    float aj = jbf.x;
    float qiqj = qi * ja.w;
    float aiaj = ai * aj;
    float u = -0.25f * r2 * (inv_ai * jbf.y);
    bool gb = u > thr;
    if (fabsf(u - thr) <= band) gb = gb_branch_exact(v.x, v.y, v.z, v.born_d, i, j, P.exp_thresh_d);
    float p14 = (bo == 3) ? P.elec14 : 1.0f;
    float S = 1.f, dSdd = 0.f;
    if (r >= P.rin) {
      float d = r - P.rin;
      float s = 1.f - P.inv_sw2 * d * d;
      dSdd = -4.f * P.inv_sw2 * d * s;
      S = s * s;
    }
    float fscal = 0.f;  // dE/dr / r for this pair (dE/d(r_i) = fscal * (p_i - p_j))
    float elec = 0.f, elf = 0.f;
    if (gb) {
      float t = __expf(u);
      float m = t * aiaj;
      float fgb = rsqrtf(r2 + m);
      float l = fgb * fgb;
      float epol = P.premul * qiqj * fgb;
      float dedr = -epol * (r - 0.25f * r * t) * l;
      float dedal = -epol * t * (1.f - u) * l;
      if (bo >= 3) {
        elec = P.econv_in * p14 * qiqj * invr;
        elf = -elec * invr;
      }
      // the switch applies to the whole GB branch (gbff.cpp:1602-1614)
      elf = S * elf + elec * dSdd;
      elec *= S;
      dedr = S * dedr + dSdd * epol;
      dedal *= S;
      epol *= S;
      fscal += dedr * 2.f * invr;
      e_pol += epol;
      deda += dedal * aj;
    } else if (bo >= 3) {
      elec = P.econv_out * p14 * qiqj * invr;
      elf = -elec * invr;
      elf = S * elf + elec * dSdd;
      elec *= S;
    }
    if (bo >= 3) {
      float vdwf = 0.f, vdw = 0.f;
      if (r < P.vdw_rc) {
        float rr = (radi + v.prm[j].x) * invr;
        float rr2 = rr * rr;
        float B = rr2 * rr2 * rr2;
        float A = B * B;
        float eps = epsi * v.prm[j].y * ((bo == 3) ? P.vdw14 : 1.0f);
        vdw = (2.f * eps) * (0.5f * A - B);
        vdwf = -(12.f * eps * invr) * (A - B);
        if (r > P.vdw_rin) {
          float d = r - P.vdw_rin;
          float s = 1.f - P.vdw_inv_sw2 * d * d;
          float ds = -4.f * P.vdw_inv_sw2 * d * s;
          s = s * s;
          vdwf = s * vdwf + vdw * ds;
          vdw *= s;
        }
      }
      e_vdw += vdw;
      e_el += elec;
      fscal += (vdwf + elf) * invr;
    }
    fx -= fscal * dx;
    fy -= fscal * dy;
    fz -= fscal * dz;
  }
  long long sx = warp_sum_ll(to_fixed_force(fx));
  long long sy = warp_sum_ll(to_fixed_force(fy));
  long long sz = warp_sum_ll(to_fixed_force(fz));
  double dv = warp_sum_d((double)e_vdw);
  double de = warp_sum_d((double)e_el);
  double dp = warp_sum_d((double)e_pol);
  double dd = warp_sum_d((double)deda);
  if (lane == 0) {
    atomicAdd((unsigned long long *)&v.fx[i], (unsigned long long)sx);
    atomicAdd((unsigned long long *)&v.fy[i], (unsigned long long)sy);
    atomicAdd((unsigned long long *)&v.fz[i], (unsigned long long)sz);
    const int N = v.n_atoms;
    double ai_d = v.born_d[i];
    double qd = (double)qi;
    double eself = P.premul_d * qd * qd / ai_d;
    v.e_atom[(size_t)AE_VDW * N + i] = 0.5 * dv;
    v.e_atom[(size_t)AE_ELEC * N + i] = 0.5 * de;
    v.e_atom[(size_t)AE_POL * N + i] = dp;
    v.e_atom[(size_t)AE_POL_SELF * N + i] = eself;
    double deda_i = dd - eself / ai_d;
    double gpi = ai_d * ai_d / 166.0;  // gbff.cpp:1755 uses the literal 166.0
    v.w_chain[i] = (float)(gpi * deda_i);
  }
}

void launch_gb_pair(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_gb_pair, (v.n_atoms + 7) / 8, 256, 0, st, v);
}

// --------------------------------------------------------------- K4 chain
__global__ void __launch_bounds__(256) k_gb_chain(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pa[i], ib = v.pb[i], ip = v.prm[i];
  const float wi = v.w_chain[i];
  const float Vi = ip.w, Ri = ip.z;
  const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
  float fx = 0.f, fy = 0.f, fz = 0.f;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    if ((ent & 7u) <= 2u) continue;
    int j = (int)(ent >> 3);
    float4 ja = v.pa[j], jb = v.pb[j];
    float dx = (ia.x - ja.x) + (ib.x - jb.x);
    float dy = (ia.y - ja.y) + (ib.y - jb.y);
    float dz = (ia.z - ja.z) + (ib.z - jb.z);
    float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > s_hi) continue;
    if (r2 > s_lo) {
      double d2 = ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]);
      if (d2 > P.still2_d) continue;
    }
    float4 jp = v.prm[j];
    float Rs = Ri + jp.z;
    float rdivR = r2 / (Rs * Rs);
    float X = 4.f;
    if (!(rdivR > P.invP5)) {
      float th = rdivR * P.piP5;
      float sn, cs;
      __sincosf(th, &sn, &cs);
      float sq = 0.5f - 0.5f * cs;
      X = 4.f * sq * sq - 2.f * sq * sn * th;
    }
    float ir2 = __frcp_rn(r2);
    float ir6 = ir2 * ir2 * ir2;
    float wj = v.w_chain[j];
    float t = P.P4 * X * ir6 * (wi * jp.w + wj * Vi);
    fx += t * dx;
    fy += t * dy;
    fz += t * dz;
  }
  long long sx = warp_sum_ll(to_fixed_force(fx));
  long long sy = warp_sum_ll(to_fixed_force(fy));
  long long sz = warp_sum_ll(to_fixed_force(fz));
  if (lane == 0) {
    atomicAdd((unsigned long long *)&v.fx[i], (unsigned long long)sx);
    atomicAdd((unsigned long long *)&v.fy[i], (unsigned long long)sy);
    atomicAdd((unsigned long long *)&v.fz[i], (unsigned long long)sz);
  }
}

void launch_gb_chain(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_gb_chain, (v.n_atoms + 7) / 8, 256, 0, st, v);
}

// --------------------------------------------------------------- Born energy
// Energy-only Born term: all pairs r <= Rc, no exp threshold, energy switch.
__global__ void __launch_bounds__(256) k_born_energy(PackView v) {
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pa[i], ib = v.pb[i];
  const float2 ab = reinterpret_cast<const float2 *>(v.born_f)[i];
  float acc = 0.f;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int j = (int)(ent >> 3);
    float4 ja = v.pa[j], jb = v.pb[j];
    float dx = (ia.x - ja.x) + (ib.x - jb.x);
    float dy = (ia.y - ja.y) + (ib.y - jb.y);
    float dz = (ia.z - ja.z) + (ib.z - jb.z);
    float r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > P.rc2) continue;
    float r = sqrtf(r2);
    float S = 1.f;
    if (!(r < P.rin)) {
      float d = r - P.rin;
      float s = 1.f - P.inv_sw2 * d * d;
      S = s * s;
    }
    float2 jbf = reinterpret_cast<const float2 *>(v.born_f)[j];
    float aiaj = ab.x * jbf.x;
    float t = __expf(-r2 * 0.25f * (ab.y * jbf.y));
    acc += S * ia.w * ja.w * rsqrtf(r2 + aiaj * t);
  }
  double sum = warp_sum_d((double)acc);
  if (lane == 0) {
    const int N = v.n_atoms;
    double ai = v.born_d[i];
    double q = (double)ia.w;
    double eself = P.premul_d * q * q / ai;
    v.e_atom[(size_t)AE_POL * N + i] = P.premul_d * sum;
    v.e_atom[(size_t)AE_POL_SELF * N + i] = eself;
  }
}

void launch_born_energy(const PackView &v, cudaStream_t st) {
  if (v.n_atoms) PDGPU_LAUNCH(k_born_energy, (v.n_atoms + 7) / 8, 256, 0, st, v);
}

// --------------------------------------------------------------- LJ/Coulomb
// FF_NonBonded fast2 kernel: all unordered pairs r <= Rc (each atom sums its
// own side, energies weighted 1/2).  Modes as selected by calcForces.
template <int EM>
__device__ __forceinline__ void nb_elec(const SysParams &P, float r, float r2, float invr, float qq,
                                        float &pot, float &frc) {
  pot = 0.f;
  frc = 0.f;
  if (EM == 1) {
    pot = P.econv_nb * qq * invr;
    frc = -pot * invr;
  } else if (EM == 2) {
    float inc = (P.dielectric + P.ddd_alpha * r) * r;
    pot = P.econv_nb * P.dielectric * qq / inc;  // econv * qq / inc
    frc = -pot * (P.dielectric + 2.f * P.ddd_alpha * r) / inc;
  } else if (EM == 3) {
    pot = P.econv_nb * qq * invr;
    frc = -pot * invr;
    if (r > P.rin) {
      float d = r - P.rin;
      float s = 1.f - P.inv_sw2 * d * d;
      float ds = -4.f * P.inv_sw2 * d * s;
      s = s * s;
      frc = s * frc + pot * ds;
      pot *= s;
    }
  } else if (EM == 4) {
    float base = P.econv_nb * qq;
    float rc2 = P.rc2, ri2 = P.rin * P.rin;
    if (r > P.rin) {
      float w = rc2 - r2;
      frc = -base * P.fs_A * invr * invr * w * w * (rc2 - 3.f * ri2 + 2.f * r2);
      pot = -base * (P.fs_A * r * (P.fs_B * invr * invr + P.fs_C + P.fs_D * r2 + P.fs_E * r2 * r2) -
                     P.fs_cutV);
    } else {
      frc = -base * invr * invr;
      pot = base * (invr - P.fs_eshift);
    }
  }
}

template <int EM>
__global__ void __launch_bounds__(256) k_nonbonded(PackView v) {
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pa[i], ib = v.pb[i], ip = v.prm[i];
  float fx = 0.f, fy = 0.f, fz = 0.f, e_vdw = 0.f, e_el = 0.f, vir = 0.f;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int bo = (int)(ent & 7u);
    if (bo < 3) continue;  // the 1-4 scaling table zeroes 1-2 and 1-3 pairs
    int j = (int)(ent >> 3);
    float4 ja = v.pa[j], jb = v.pb[j];
    float dx = (ia.x - ja.x) + (ib.x - jb.x);
    float dy = (ia.y - ja.y) + (ib.y - jb.y);
    float dz = (ia.z - ja.z) + (ib.z - jb.z);
    float r2 = dx * dx + dy * dy + dz * dz;
    if (EM == 1 || EM == 2) {
      // unswitched Coulomb is discontinuous at Rc: decide boundary pairs
      // with the reference's FP64 expression (fv = p_j - p_i; innerdot)
      if (fabsf(r2 - P.rc2) <= 4e-6f * P.rc2) {
        double d2 = ref_d2(v.x[j], v.y[j], v.z[j], v.x[i], v.y[i], v.z[i]);
        if (d2 > P.rc2_d) continue;
      } else if (r2 > P.rc2) {
        continue;
      }
    } else if (r2 > P.rc2) {
      continue;
    }
    float invr = rsqrtf(r2);
    float r = r2 * invr;
    float vdw = 0.f, vdwf = 0.f;
    if (P.vdw_mode && r < P.vdw_rc) {
      float4 jp = v.prm[j];
      float rr = (ip.x + jp.x) * invr;
      float rr2 = rr * rr;
      float B = rr2 * rr2 * rr2;
      float A = B * B;
      float eps = ((bo == 3) ? P.vdw14 : 1.f) * ip.y * jp.y;
      vdw = (2.f * eps) * (0.5f * A - B);
      vdwf = -(12.f * eps * invr) * (A - B);
      if (r > P.vdw_rin) {
        float d = r - P.vdw_rin;
        float s = 1.f - P.vdw_inv_sw2 * d * d;
        float ds = -4.f * P.vdw_inv_sw2 * d * s;
        s = s * s;
        vdwf = s * vdwf + vdw * ds;
        vdw *= s;
      }
    }
    float pot, frc;
    float qq = ia.w * ja.w * ((bo == 3) ? P.elec14 : 1.f);
    nb_elec<EM>(P, r, r2, invr, qq, pot, frc);
    float fm = vdwf + frc;
    e_vdw += vdw;
    e_el += pot;
    vir += r * fm;
    float s = fm * invr;  // force on i along (p_j - p_i): f_i += s * (p_j - p_i)
    fx -= s * dx;
    fy -= s * dy;
    fz -= s * dz;
  }
  long long sx = warp_sum_ll(to_fixed_force(fx));
  long long sy = warp_sum_ll(to_fixed_force(fy));
  long long sz = warp_sum_ll(to_fixed_force(fz));
  double dv = warp_sum_d((double)e_vdw);
  double de = warp_sum_d((double)e_el);
  double dw = warp_sum_d((double)vir);
  if (lane == 0) {
    atomicAdd((unsigned long long *)&v.fx[i], (unsigned long long)sx);
    atomicAdd((unsigned long long *)&v.fy[i], (unsigned long long)sy);
    atomicAdd((unsigned long long *)&v.fz[i], (unsigned long long)sz);
    const int N = v.n_atoms;
    v.e_atom[(size_t)AE_VDW * N + i] = 0.5 * dv + P.vdwcor_e_d;
    v.e_atom[(size_t)AE_ELEC * N + i] = 0.5 * de;
    v.e_atom[(size_t)AE_VIR * N + i] = 0.5 * dw;
  }
}

void launch_nonbonded(const PackView &v, cudaStream_t st, int elec_mode) {
  if (!v.n_atoms) return;
  // the mode is per system; a pack holds systems of one mode (checked when
  // the pack is built)
  int blocks = (v.n_atoms + 7) / 8;
  switch (elec_mode) {
    case 0: PDGPU_LAUNCH((k_nonbonded<0>), blocks, 256, 0, st, v); break;
    case 1: PDGPU_LAUNCH((k_nonbonded<1>), blocks, 256, 0, st, v); break;
    case 2: PDGPU_LAUNCH((k_nonbonded<2>), blocks, 256, 0, st, v); break;
    case 3: PDGPU_LAUNCH((k_nonbonded<3>), blocks, 256, 0, st, v); break;
    default: PDGPU_LAUNCH((k_nonbonded<4>), blocks, 256, 0, st, v); break;
  }
}

// --------------------------------------------------------------- pair counts
// Instrumentation: the pair sets the roofline counts use, decided exactly as
// the kernels decide them.  out[0] P_B (directed, r <= still cutoff, bo >= 3),
// out[1] P_H (unordered, r <= Rc), out[2] list entries.
__global__ void k_pair_counts(PackView v, unsigned long long *out) {
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (i >= v.n_atoms) return;
  const SysParams &P = v.sp[v.sys_of[i]];
  const float4 ia = v.pa[i], ib = v.pb[i];
  unsigned long long pb = 0, ph = 0;
  long long b = v.row_start[i], e = v.row_start[i + 1];
  for (long long k = b + lane; k < e; k += 32) {
    unsigned ent = v.nl[k];
    int j = (int)(ent >> 3);
    float4 ja = v.pa[j], jb = v.pb[j];
    float dx = (ia.x - ja.x) + (ib.x - jb.x);
    float dy = (ia.y - ja.y) + (ib.y - jb.y);
    float dz = (ia.z - ja.z) + (ib.z - jb.z);
    float r2 = dx * dx + dy * dy + dz * dz;
    if (j < i && r2 <= P.rc2) ph++;
    if ((ent & 7u) > 2u && ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) <= P.still2_d) pb++;
  }
  for (int o = 16; o > 0; o >>= 1) {
    pb += __shfl_xor_sync(0xffffffffu, pb, o);
    ph += __shfl_xor_sync(0xffffffffu, ph, o);
  }
  if (lane == 0) {
    atomicAdd(&out[0], pb);
    atomicAdd(&out[1], ph);
    atomicAdd(&out[2], (unsigned long long)(e - b));
  }
}

void launch_pair_counts(const PackView &v, cudaStream_t st, unsigned long long *out) {
  if (v.n_atoms) PDGPU_LAUNCH(k_pair_counts, (v.n_atoms + 7) / 8, 256, 0, st, v, out);
}

}  // namespace pdgpu
