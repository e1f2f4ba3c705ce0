// FF_SASA_LCPO: the LCPO surface-area term (Weiser, Shenkin & Still,
// J. Comp. Chem. 20:217, 1999) as forcefields/lcpo.cpp evaluates it, with
// the reference's neighbour list, its 80-partner overlap lists and its
// UpdateSasa cadence.
//
// Two launches per evaluation, one warp per atom the term uses (hydrogens,
// use 0, keep area, energy and derivative 0 and get no warp):
//  k_lcpo_list  the atom's overlap partners: the list partners j with
//               use[j] and |xi - xj| < ri + rj (from its CSR row, or from
//               the candidates k_lcpo_cand_tiles gathered off the tiles of a
//               tile search), ranked by index, the first 80 kept with their
//               overlap areas.  The reference appends
//               partners in ascending index from both ends of every pair
//               and stops at 80 (lcpo.cpp:434-485, 688-746), which keeps
//               exactly these.
//  k_lcpo_eval  the atom's area and SASAderiv (lcpo.cpp:751-941): lane e
//               takes partner e and runs its inner loop over the partner's
//               own list in the reference's order; the per-partner terms go
//               to shared memory and twelve lanes then add them in partner
//               order, one accumulator each, so every sum has the
//               reference's rounding.  The file is compiled without fused
//               multiply-adds (build.py), so the FP64 arithmetic matches
//               the reference compiled without contraction bit for bit.
// A system whose step is not due (Step % UpdateSasa != 0) adds the
// derivative it holds from its last full evaluation (lcpo.cpp:641-659).
// Units: areas A^2, sigma kcal/mol/A^2, SASAderiv kcal/mol/A.
#include <cuda_runtime.h>

#include "internal.cuh"

namespace pdgpu {

constexpr int kLcpoWarps = 4;    // atoms per block
constexpr int kLcpoQ = 14;       // per-partner terms kept for the ordered sums
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kFourPi = 4.0 * kPi;

__device__ __forceinline__ bool lcpo_due(const LcpoView &lc, const StepSrc &ss, int s) {
  const int step = ss.p ? __ldcg(ss.p + (size_t)s * ss.stride) : ss.imm;
  return step % lc.update == 0;
}

// The overlap test of a pair, from either end: the force path compares
// d^2 with (ri + rj)^2 (lcpo.cpp:713), the energy path d with ri + rj
// (lcpo.cpp:460); d^2 takes the same value from both ends.
template <bool EO>
__device__ __forceinline__ bool lcpo_overlaps(double d2, double rs) {
  return EO ? sqrt(d2) < rs : d2 < rs * rs;
}

// Overlap candidates from the tiles of the last tile search: each list pair
// (one tile bit, stored once) that overlaps is appended to both atoms'
// candidate buffers; k_lcpo_list ranks them, so the order of the appends
// does not matter.  A warp takes one tile at a time, lane l for the
// i-cluster's atom l, over a contiguous range of the tiles: an i-cluster's
// tiles sit together in the store, so warps that run at once append to
// different atoms' counters instead of all to the same 32.
template <bool EO>
__global__ void __launch_bounds__(128) k_lcpo_cand_tiles(PackView v, StepSrc ss) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const LcpoView &lc = v.lc;
  const int lane = threadIdx.x & 31;
  const long long T = v.tile_count[0];
  const long long W = (long long)gridDim.x * (blockDim.x >> 5);
  const long long g = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int e_end = (int)(T * (g + 1) / W);
  for (int e = (int)(T * g / W); e < e_end; e++) {
    const int4 m = v.tile_meta[e];
    const int s = m.w >> 8, na = ((m.w >> 3) & 31) + 1, nb = (m.w & 7) + 1;
    if (!EO && !lcpo_due(lc, ss, s)) continue;
    if (lane >= na) continue;
    const int i = m.z + lane;
    unsigned row = reinterpret_cast<const unsigned char *>(v.tile_rows)[32 * (size_t)e + lane];
    if (!row || !lc.use[i]) continue;
    const double4 pi = v.xyzp[i];
    const double ri = lc.r[i];
    for (int t = 0; t < nb; t++) {
      if (!((row >> t) & 1u)) continue;
      const int j = m.x + t;
      if (!lc.use[j]) continue;
      const double4 pj = v.xyzp[j];
      const double g = pi.x - pj.x, h = pi.y - pj.y, k = pi.z - pj.z;
      if (!lcpo_overlaps<EO>(g * g + h * h + k * k, ri + lc.r[j])) continue;
      const int qi = atomicAdd(&lc.cand_n[i], 1);
      if (qi < kLcpoCand) lc.cand[(size_t)i * kLcpoCand + qi] = j;
      const int qj = atomicAdd(&lc.cand_n[j], 1);
      if (qj < kLcpoCand) lc.cand[(size_t)j * kLcpoCand + qj] = i;
    }
  }
}

template <bool EO, bool TILES>
__global__ void __launch_bounds__(kLcpoWarps * 32) k_lcpo_list(PackView v, StepSrc ss) {
  __shared__ int cand[kLcpoWarps][kLcpoCand];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const LcpoView &lc = v.lc;
  const int w = blockIdx.x * kLcpoWarps + warp;
  if (w >= lc.n_used || v.flags[F_NL_OVERFLOW]) return;
  const int i = lc.atoms[w];
  if (!EO && !lcpo_due(lc, ss, v.sys_of[i])) return;
  if (!lc.use[i]) {
    if (lane == 0) lc.cnt[i] = 0;
    return;
  }
  const double4 pi = v.xyzp[i];  // (x, y, z) as in v.x, v.y, v.z
  const double xi = pi.x, yi = pi.y, zi = pi.z, ri = lc.r[i];
  if (lane == 0) lc.xr[i] = make_double4(xi, yi, zi, ri);  // for the evaluation's gathers
  int n = 0;
  if (TILES) {
    n = lc.cand_n[i];
    for (int q = lane; q < min(n, kLcpoCand); q += 32) cand[warp][q] = lc.cand[(size_t)i * kLcpoCand + q];
    __syncwarp();
    if (lane == 0) lc.cand_n[i] = 0;  // clean for the next evaluation
  } else {
    const long long r0 = v.row_start[i];
    const int rn = v.row_cnt[i];
    for (int q0 = 0; q0 < rn; q0 += 32) {
      const int q = q0 + lane;
      bool hit = false;
      int j = 0;
      if (q < rn) {
        j = (int)(v.nl[r0 + q] >> 3);
        if (lc.use[j]) {
          const double4 pj = v.xyzp[j];
          const double g = xi - pj.x, h = yi - pj.y, k = zi - pj.z;
          hit = lcpo_overlaps<EO>(g * g + h * h + k * k, ri + lc.r[j]);
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      const int at = n + __popc(m & ((1u << lane) - 1u));
      if (hit && at < kLcpoCand) cand[warp][at] = j;
      n += __popc(m);
    }
  }
  if (n > kLcpoCand) {
    if (lane == 0) atomicExch(&v.flags[F_LCPO_CAND], 1);
    n = kLcpoCand;
  }
  __syncwarp();
  if (lane == 0) lc.cnt[i] = min(n, kLcpoMax);
  const size_t base = (size_t)i * kLcpoMax;
  for (int q = lane; q < n; q += 32) {
    const int j = cand[warp][q];
    int rank = 0;
    for (int t = 0; t < n; t++) rank += cand[warp][t] < j;
    if (rank >= kLcpoMax) continue;
    const double4 pj = v.xyzp[j];
    const double g = xi - pj.x, h = yi - pj.y, k = zi - pj.z;
    const double d = sqrt(g * g + h * h + k * k);
    const double rj = lc.r[j];
    double s;
    if (EO) {
      // sphereSurfaceOverlap(ri, rj, d) (maths/maths.cpp:103-106), >= 0
      s = kTwoPi * ri * (ri - d / 2.0 - (ri * ri - rj * rj) / (2.0 * d));
      if (s < 0) s = 0;
    } else {
      // sij of lcpo.cpp:716-718; from the other end of the pair the same
      // expression with the half-difference negated, which is this one
      const double hd = 0.5 * (ri * ri - rj * rj) * (1 / d);
      s = kTwoPi * ri * (ri - d * 0.5 - hd);
    }
    lc.idx[base + rank] = j;
    lc.s[base + rank] = s;
  }
}

__device__ __forceinline__ void lcpo_add_force(const PackView &v, int i, double fx, double fy, double fz) {
  atomicAdd((unsigned long long *)&v.fx[i], (unsigned long long)__double2ll_rn(fx * kForceScale));
  atomicAdd((unsigned long long *)&v.fy[i], (unsigned long long)__double2ll_rn(fy * kForceScale));
  atomicAdd((unsigned long long *)&v.fz[i], (unsigned long long)__double2ll_rn(fz * kForceScale));
}

// per-partner terms in shared memory: 0-2 dSASA_2 (scaled by P2 sigma of
// the partner), 3-5 dSASA_3, 6-8 dSASA_4, 9 Si2_t, 10 Si3_t, 11-13
// dAijdc_2t; a row per term, padded so the twelve summing lanes read
// different banks
template <bool EO>
__global__ void __launch_bounds__(kLcpoWarps * 32) k_lcpo_eval(PackView v, StepSrc ss) {
  __shared__ double T[kLcpoWarps][kLcpoQ][kLcpoMax + 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const LcpoView &lc = v.lc;
  const int w = blockIdx.x * kLcpoWarps + warp;
  if (w >= lc.n_used || v.flags[F_NL_OVERFLOW]) return;
  const int i = lc.atoms[w];
  const size_t N = (size_t)v.n_atoms;
  if (!EO && !lcpo_due(lc, ss, v.sys_of[i])) {
    // the held step: the energy and forces of the last full evaluation
    // (lcpo.cpp:641-659 adds SASA * sigma and SASAderiv again), written
    // afresh so that a zeroed record (WorkSpace::zeroForces) holds them too
    if (lane == 0) {
      v.e_atom[AE_SURF * N + i] = lc.sasa[i] * lc.sigma[i];
      const double dx = lc.deriv[i], dy = lc.deriv[N + i], dz = lc.deriv[2 * N + i];
      if (dx != 0.0 || dy != 0.0 || dz != 0.0) lcpo_add_force(v, i, dx, dy, dz);
    }
    return;
  }
  if (!lc.use[i]) {
    if (lane == 0) {
      lc.sasa[i] = 0.0;
      v.e_atom[AE_SURF * N + i] = 0.0;
      if (!EO) lc.deriv[i] = lc.deriv[N + i] = lc.deriv[2 * N + i] = 0.0;
    }
    return;
  }
  double(*W)[kLcpoMax + 1] = T[warp];
  const double4 pi4 = lc.xr[i];
  const double xi = pi4.x, yi = pi4.y, zi = pi4.z, ri = pi4.w;
  const int cnt = lc.cnt[i];
  const size_t base = (size_t)i * kLcpoMax;
  for (int e = lane; e < cnt; e += 32) {
    const int ja = lc.idx[base + e];
    const double si2 = lc.s[base + e];
    const int nj = lc.cnt[ja];
    const size_t jb = (size_t)ja * kLcpoMax;
    double si3 = 0.0;
    if (EO) {
      // lcpo.cpp:517-537
      for (int k = 0; k < nj; k++) {
        const int ka = lc.idx[jb + k];
        if (ka == i) continue;
        const double4 pk = lc.xr[ka];
        const double g = pk.x - xi, h = pk.y - yi, q = pk.z - zi;
        if (ri + pk.w < sqrt(g * g + h * h + q * q)) continue;
        si3 += lc.s[jb + k];
      }
    } else {
      // lcpo.cpp:772-901
      const double4 pj4 = lc.xr[ja];
      const double xj = pj4.x, yj = pj4.y, zj = pj4.z, rj = pj4.w;
      const double gx = xj - xi, gy = yj - yi, gz = zj - zi;
      const double dij = sqrt(gx * gx + gy * gy + gz * gz);
      const double invij = 1 / dij;
      double hd = 0.5 * (ri * ri - rj * rj) * invij;
      const double sji = kTwoPi * rj * (rj - dij * 0.5 + hd);
      hd *= 2.0 * invij;
      const double ddx = -(xi - xj) / dij, ddy = -(yi - yj) / dij, ddz = -(zi - zj) / dij;
      double dAdd = kPi * rj * (-hd - 1);
      double d2x = dAdd * ddx, d2y = dAdd * ddy, d2z = dAdd * ddz;
      dAdd = kPi * ri * (hd - 1);
      const double a2x = dAdd * ddx, a2y = dAdd * ddy, a2z = dAdd * ddz;
      double d3x = 0, d3y = 0, d3z = 0, d3bx = 0, d3by = 0, d3bz = 0, d4bx = 0, d4by = 0, d4bz = 0;
      double s3ik = 0.0;
      // the next partner's index, record and overlap are loaded one
      // iteration ahead
      int kn = nj > 0 ? lc.idx[jb] : 0;
      double4 pn = nj > 0 ? lc.xr[kn] : make_double4(0, 0, 0, 0);
      double sn = nj > 0 ? lc.s[jb] : 0.0;
      for (int k = 0; k < nj; k++) {
        const int ka = kn;
        const double xk = pn.x, yk = pn.y, zk = pn.z, rk = pn.w;
        const double sjk = sn;
        if (k + 1 < nj) {
          kn = lc.idx[jb + k + 1];
          pn = lc.xr[kn];
          sn = lc.s[jb + k + 1];
        }
        if (ka == i) continue;
        const double g = xk - xi, h = yk - yi, q = zk - zi;
        double dik = g * g + h * h + q * q;
        if ((ri + rk) * (ri + rk) < dik) continue;
        dik = sqrt(dik);
        const double invik = 1 / dik;
        const double hk = (ri * ri - rk * rk) * (invik * invik);
        dAdd = kPi * ri * (hk - 1);
        const double dkx = -(xi - xk) * invik, dky = -(yi - yk) * invik, dkz = -(zi - zk) * invik;
        d3x += dAdd * dkx;
        d3y += dAdd * dky;
        d3z += dAdd * dkz;
        dAdd = kPi * rk * (-hk - 1);
        s3ik += kPi * ri * (2 * ri - dik - dik * hk);
        d3bx += dAdd * dkx;
        d3by += dAdd * dky;
        d3bz += dAdd * dkz;
        d4bx += sjk * dAdd * dkx;
        d4by += sjk * dAdd * dky;
        d4bz += sjk * dAdd * dkz;
        si3 += sjk;
      }
      double d4x = sji * d3x + d4bx, d4y = sji * d3y + d4by, d4z = sji * d3z + d4bz;
      d3x += d3bx;
      d3y += d3by;
      d3z += d3bz;
      d4x += d2x * s3ik;
      d4y += d2y * s3ik;
      d4z += d2z * s3ik;
      const double4 pj = lc.p[ja];
      const double sj = lc.sigma[ja];
      const double m2 = pj.y * sj, m3 = pj.z * sj, m4 = pj.w * sj;
      W[0][e] = d2x * m2;
      W[1][e] = d2y * m2;
      W[2][e] = d2z * m2;
      W[3][e] = d3x * m3;
      W[4][e] = d3y * m3;
      W[5][e] = d3z * m3;
      W[6][e] = d4x * m4;
      W[7][e] = d4y * m4;
      W[8][e] = d4z * m4;
      W[11][e] = a2x;
      W[12][e] = a2y;
      W[13][e] = a2z;
    }
    W[9][e] = si2;
    W[10][e] = si3;
  }
  __syncwarp();
  // ordered sums over the partners (lcpo.cpp:903-920): lanes 0-2 SASAderiv
  // x y z, 3 Si4, 4 Si3, 5 Si2, 6-8 dAijdc_2, 9-11 dAijdc_4
  double acc = 0.0;
  if (lane < 3) {
    if (!EO)
      for (int e = 0; e < cnt; e++) {
        acc += W[lane][e];
        acc += W[3 + lane][e];
        acc += W[6 + lane][e];
      }
  } else if (lane == 3) {
    for (int e = 0; e < cnt; e++) acc += W[10][e] * W[9][e];
  } else if (lane == 4) {
    for (int e = 0; e < cnt; e++) acc += W[10][e];
  } else if (lane == 5) {
    for (int e = 0; e < cnt; e++) acc += W[9][e];
  } else if (lane < 9) {
    if (!EO)
      for (int e = 0; e < cnt; e++) acc += W[5 + lane][e];
  } else if (lane < 12) {
    if (!EO)
      for (int e = 0; e < cnt; e++) acc += W[10][e] * W[2 + lane][e];
  }
  double R[12];
#pragma unroll
  for (int c = 0; c < 12; c++) R[c] = __shfl_sync(0xffffffffu, acc, c);
  if (lane != 0) return;
  const double4 pi = lc.p[i];
  const double sig = lc.sigma[i];
  const double Si = kFourPi * ri * ri;  // sphereSurfaceArea (maths/maths.cpp:97-100)
  double SAi = pi.x * Si + pi.y * R[5] + pi.z * R[4] + pi.w * R[3];
  double D[3] = {R[0], R[1], R[2]};
  if (!EO) {
    const double m2 = pi.y * sig, m4 = pi.w * sig;
    for (int c = 0; c < 3; c++) D[c] += R[6 + c] * m2;
    for (int c = 0; c < 3; c++) D[c] += R[9 + c] * m4;
  }
  if (SAi < 0) {  // lcpo.cpp:926-929
    SAi = 0;
    D[0] = D[1] = D[2] = 0.0;
  }
  lc.sasa[i] = SAi;
  v.e_atom[AE_SURF * N + i] = SAi * sig;
  if (!EO) {
    lc.deriv[i] = D[0];
    lc.deriv[N + i] = D[1];
    lc.deriv[2 * N + i] = D[2];
    if (D[0] != 0.0 || D[1] != 0.0 || D[2] != 0.0) lcpo_add_force(v, i, D[0], D[1], D[2]);
  }
}

void launch_lcpo_part(const PackView &v, cudaStream_t st, StepSrc step, bool energy_only, bool from_tiles,
                      int part) {
  if (v.lc.update <= 0 || !v.lc.n_used) return;
  const int blocks = (v.lc.n_used + kLcpoWarps - 1) / kLcpoWarps;
  const int tpb = kLcpoWarps * 32;
  if (part == 0) {
    if (from_tiles) {
      static int sms = 0;  // a persistent grid: eight 4-warp blocks per SM
      if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
      }
      if (energy_only)
        PDGPU_LAUNCH(k_lcpo_cand_tiles<true>, 8 * sms, 128, 0, st, v, step);
      else
        PDGPU_LAUNCH(k_lcpo_cand_tiles<false>, 8 * sms, 128, 0, st, v, step);
    }
    if (energy_only) {
      if (from_tiles)
        PDGPU_LAUNCH((k_lcpo_list<true, true>), blocks, tpb, 0, st, v, step);
      else
        PDGPU_LAUNCH((k_lcpo_list<true, false>), blocks, tpb, 0, st, v, step);
    } else {
      if (from_tiles)
        PDGPU_LAUNCH((k_lcpo_list<false, true>), blocks, tpb, 0, st, v, step);
      else
        PDGPU_LAUNCH((k_lcpo_list<false, false>), blocks, tpb, 0, st, v, step);
    }
  } else {
    if (energy_only)
      PDGPU_LAUNCH(k_lcpo_eval<true>, blocks, tpb, 0, st, v, step);
    else
      PDGPU_LAUNCH(k_lcpo_eval<false>, blocks, tpb, 0, st, v, step);
  }
}
void launch_lcpo(const PackView &v, cudaStream_t st, StepSrc step, bool energy_only, bool from_tiles) {
  launch_lcpo_part(v, st, step, energy_only, from_tiles, 0);
  launch_lcpo_part(v, st, step, energy_only, from_tiles, 1);
}

}  // namespace pdgpu
