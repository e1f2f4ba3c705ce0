// Cluster-pair tiles: the neighbour pair set re-cut into 32 x 8 blocks so
// the three pair passes read their partners once per block with coalesced
// loads and evaluate each unordered pair once.
//
// Atoms of a system are cut, in their own order (residue order: bonded and
// spatially close atoms are neighbours in memory), into i-clusters of 32
// (one per lane of a warp) and j-clusters of 8.  The tiles of an i-cluster
// are the j-clusters at or after it that hold a list partner of one of its
// atoms; they are read off the neighbour list itself (built with the
// reference's FP64 predicate, neighbourlist.cpp:263-266), so a tile's bits
// are exactly list pairs: every unordered list pair sits in one tile (the
// pair with j > i where the j-cluster lies inside the i-cluster).  A tile
// stores, per i lane, one byte of bits over its 8 j atoms; tiles with 1-2,
// 1-3 or 1-4 partners (bond orders from the list entries) carry two more
// byte rows: bond order <= 2 and bond order == 3.
//
// Each pass runs one block per i-cluster; its warps take the cluster's
// tiles in turn, prefetching the next tile's 8 j atoms while they work on
// the current one.  Lane l = 8g + a (one i atom) walks the tile's j atoms in
// the order (a+t) mod 8: the i side accumulates in registers, the j side
// goes with one shuffle to the lane of its group that owns the j atom; after
// the 8 steps the four groups' j sums meet with two xor shuffles and are
// added to the j atoms with 64-bit fixed-point atomics (order-independent).
// Per-lane i sums are added in fixed warp order.  Pass results:
//   K2 k_born_tile   Born sums, i and j side, fixed point 2^40 (exact);
//                    k_born_finish inverts them (FP64) and zeroes the j-side
//                    accumulators of the next passes
//   K3 k_gb_tile     forces (i: FP64 pair force, j: fixed point 2^24),
//                    per-atom LJ / Coulomb / GB energies and dE/da (i side
//                    FP64, j side fixed point); k_gb_finish forms the
//                    reference's per-atom values and the chain-rule weights
//   K4 k_chain_tile  chain-rule forces (i and j side as K3)
// The per-pair arithmetic is the row kernels' (pairmath.cuh).
#include <cuda_runtime.h>

#include "pairmath.cuh"

namespace pdgpu {

constexpr int kTileWarps = 4;    // warps per block (one block per i-cluster)
constexpr int kBuildChunk = 128; // tiles assembled in shared memory at a time

// --------------------------------------------------------------- tile list
// One block per i-cluster.  (1) A bitmap over the system's j-clusters at or
// after the i-cluster marks those holding a half-list partner; (2) its set
// bits, in order, are the cluster's tiles (deterministic order); (3) the
// rows are scanned again to set the pair bits and the bond-order bits of
// each tile, kBuildChunk tiles at a time in shared memory.
__device__ __forceinline__ bool half_pair(int i, int j, int a0) {
  // j in a later j-cluster, or in this i-cluster with j > i
  return j >= a0 && (j >= a0 + 32 || j > i);
}

__global__ void __launch_bounds__(128) k_tile_build(PackView v) {
  extern __shared__ unsigned sm[];
  const int sc = blockIdx.x;
  if (v.flags[F_NL_OVERFLOW]) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = v.sc_sys[sc];
  const int a0 = v.sc_atom0[sc];
  const int end = v.atom_off[s + 1];
  const int na = min(32, end - a0);
  const int nbits = (end - a0 + 7) / 8;  // j-clusters at or after a0
  const int W = (nbits + 31) / 32;
  unsigned *bm = sm;                                // [W]
  unsigned *pre = bm + W;                           // [W+1]
  int *cb0 = (int *)(pre + W + 1);                  // [chunk] first j atom
  unsigned *rw = (unsigned *)(cb0 + kBuildChunk);   // [chunk*8] pair bits: byte l of word l/4
  unsigned *xw = rw + kBuildChunk * 8;              // bond order <= 2
  unsigned *bw = xw + kBuildChunk * 8;              // bond order == 3
  __shared__ int base_s;
  for (int w = tid; w < W; w += blockDim.x) bm[w] = 0;
  __syncthreads();
  for (int q = warp; q < na; q += kTileWarps) {
    const int i = a0 + q;
    const long long b = v.row_start[i], e = v.row_start[i + 1];
    for (long long k = b + lane; k < e; k += 32) {
      const int j = (int)(v.nl[k] >> 3);
      if (half_pair(i, j, a0)) {
        const int p = (j - a0) >> 3;
        atomicOr(&bm[p >> 5], 1u << (p & 31));
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    int c = 0;
    for (int w = 0; w < W; w++) {
      pre[w] = c;
      c += __popc(bm[w]);
    }
    pre[W] = c;
    base_s = atomicAdd(&v.tile_count[0], c);
  }
  __syncthreads();
  const int ncand = pre[W];
  const int base = base_s;
  if ((long long)base + ncand > v.tile_cap) {  // cannot happen: the capacity is the worst case
    if (tid == 0) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
    return;
  }
  for (int c0 = 0; c0 < ncand; c0 += kBuildChunk) {
    for (int w = tid; w < kBuildChunk * 8 * 3; w += blockDim.x) rw[w] = 0;
    for (int w = tid; w < W; w += blockDim.x) {
      unsigned bits = bm[w];
      while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1;
        const int r = pre[w] + __popc(bm[w] & ((1u << b) - 1u)) - c0;
        if (r >= 0 && r < kBuildChunk) cb0[r] = a0 + 8 * (32 * w + b);
      }
    }
    __syncthreads();
    for (int q = warp; q < na; q += kTileWarps) {
      const int i = a0 + q;
      const long long b = v.row_start[i], e = v.row_start[i + 1];
      for (long long k = b + lane; k < e; k += 32) {
        const unsigned ent = v.nl[k];
        const int j = (int)(ent >> 3);
        if (!half_pair(i, j, a0)) continue;
        const int p = (j - a0) >> 3;
        const int r = pre[p >> 5] + __popc(bm[p >> 5] & ((1u << (p & 31)) - 1u)) - c0;
        if (r < 0 || r >= kBuildChunk) continue;
        const unsigned bit = 1u << ((q & 3) * 8 + ((j - a0) & 7));
        const int wi = r * 8 + (q >> 2);
        atomicOr(&rw[wi], bit);
        const unsigned bo = ent & 7u;
        if (bo <= 2u) atomicOr(&xw[wi], bit);
        if (bo == 3u) atomicOr(&bw[wi], bit);
      }
    }
    __syncthreads();
    const int nr = min(kBuildChunk, ncand - c0);
    for (int r = tid; r < nr; r += blockDim.x) {
      const int et = base + c0 + r;
      v.tile_b0[et] = cb0[r];
      unsigned spec_any = 0;
      for (int w = 0; w < 8; w++) {
        v.tile_rows[8 * (size_t)et + w] = rw[r * 8 + w];
        spec_any |= xw[r * 8 + w] | bw[r * 8 + w];
      }
      int spec = -1;
      if (spec_any) {
        spec = atomicAdd(&v.tile_count[1], 1);
        if (spec < v.spec_cap) {
          for (int w = 0; w < 8; w++) {
            v.spec_rows[16 * (size_t)spec + w] = xw[r * 8 + w];
            v.spec_rows[16 * (size_t)spec + 8 + w] = bw[r * 8 + w];
          }
        } else {
          atomicExch(&v.flags[F_NL_OVERFLOW], 1);
          spec = -1;
        }
      }
      v.tile_spec[et] = spec;
    }
    __syncthreads();
  }
  if (tid == 0) {
    v.tile_e0[sc] = base;
    v.tile_e1[sc] = base + ncand;
  }
}

// --------------------------------------------------------------- tile passes
__device__ __forceinline__ long long to_fixed_j(float f) {
  // saturate far outside any physical range (clashing trial structures
  // stay well inside: 2^39 kcal/mol/A)
  float s = fminf(fmaxf(f * (float)kJScale, -9.0e18f), 9.0e18f);
  return __float2ll_rn(s);
}

// A lane's row bits of tile e (bits over the 8 j atoms), and of its
// bond-order rows when the tile has them.
__device__ __forceinline__ unsigned tile_row(const PackView &v, int e, int lane) {
  return reinterpret_cast<const unsigned char *>(v.tile_rows)[32 * (size_t)e + lane];
}
__device__ __forceinline__ unsigned spec_row(const PackView &v, int spec, int which, int lane) {
  return reinterpret_cast<const unsigned char *>(v.spec_rows)[64 * (size_t)spec + 32 * which + lane];
}

// Staging of a tile's j atoms: lanes 0..7 hold three records of their j
// atom in registers (prefetched one tile ahead) and write them to the
// warp's shared slots before the tile is processed.
struct JStage {
  float4 a, b, c;
  int b0, nb, spec;
  unsigned row;
};
template <int REC>  // third record: 0 chainp (radius R, volume V, chain weight w), 1 prm (LJ radius, eps)
__device__ __forceinline__ void stage_load(const PackView &v, int e, int end, int lane, JStage &q) {
  q.b0 = v.tile_b0[e];
  q.nb = min(8, end - q.b0);
  q.spec = v.tile_spec[e];
  q.row = tile_row(v, e, lane);
  if (lane < q.nb) {
    const int j = q.b0 + lane;
    q.a = v.pq[2 * (size_t)j];
    q.b = v.pq[2 * (size_t)j + 1];
    q.c = REC == 0 ? v.chainp[j] : v.prm[j];
  }
}

// --------------------------------------------------------------- K2 tiles
// (register bounds: five blocks per SM, one wave for a 20k-atom system)
__global__ void __launch_bounds__(32 * kTileWarps, 5) k_born_tile(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane & ~7, a = lane & 7;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sC[kTileWarps][8];
  const int s = v.sc_sys[sc];
  const SysParams &P = v.sp[s];
  const int a0 = v.sc_atom0[sc];
  const int end = v.atom_off[s + 1];
  const int na = min(32, end - a0);
  const int i = a0 + (lane < na ? lane : 0);
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ic = v.chainp[i];
  const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
  const float invP5 = P.invP5, piP5 = P.piP5, P4s = P.P4 * (float)kBornScale;
  const double still2_d = P.still2_d;
  long long acc_i = 0;
  const int e1 = v.tile_e1[sc];
  int e = v.tile_e0[sc] + warp;
  JStage nx;
  if (e < e1) stage_load<0>(v, e, end, lane, nx);
  while (e < e1) {
    const JStage cur = nx;
    if (lane < cur.nb) {
      sA[warp][lane] = cur.a;
      sB[warp][lane] = cur.b;
      sC[warp][lane] = cur.c;
    }
    unsigned rows = cur.row;
    if (cur.spec >= 0) rows &= ~spec_row(v, cur.spec, 0, lane);  // bond order > 2 only
    __syncwarp();
    const int en = e + kTileWarps;
    if (en < e1) stage_load<0>(v, en, end, lane, nx);
    long long jacc = 0;  // lane (g,a): j atom a, this group's i atoms
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const int jt = (a + t) & 7;
      long long ti = 0, tj = 0;
      if ((rows >> jt) & 1u) {
        const float4 ja = sA[warp][jt], jb = sB[warp][jt], jc = sC[warp][jt];
        const Dx d = diff(ia, ib, ja, jb);
        bool ok = d.r2 <= s_lo;
        if (!ok && d.r2 <= s_hi) {
          const int j = cur.b0 + jt;
          ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) > still2_d);
        }
        if (ok) {
          const float term = born_term_noV(d, ic.x, jc.x, invP5, piP5, P4s);
          ti = __float2ll_rn(__fmul_rn(term, jc.y));
          tj = __float2ll_rn(__fmul_rn(term, ic.y));
        }
      }
      acc_i += ti;
      jacc += __shfl_sync(0xffffffffu, tj, g8 | ((a - t) & 7));
    }
    jacc += __shfl_xor_sync(0xffffffffu, jacc, 8);
    jacc += __shfl_xor_sync(0xffffffffu, jacc, 16);
    if (lane < cur.nb && jacc) atomicAdd((unsigned long long *)&v.bsum[cur.b0 + lane], (unsigned long long)jacc);
    __syncwarp();
    e = en;
  }
  if (lane < na && acc_i) atomicAdd((unsigned long long *)&v.bsum[a0 + lane], (unsigned long long)acc_i);
}

// a_i = -halfeconv / (terms123_i + sum) (FP64); zero the accumulators the
// following passes add into (and, first in an evaluation, the forces)
__global__ void k_born_finish(PackView v, int zero_first) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  const int s = v.sys_of[i];
  const SysParams &P = v.sp[s];
  long long sum = v.bsum[i];
  v.bsum[i] = 0;
  double Gpol = v.terms123[i] + (double)sum * kInvBornScale;
  double a = -P.halfeconv_d / Gpol + P.born_offset_d;
  v.born_d[i] = a;
  reinterpret_cast<float *>(&v.pq[2 * (size_t)i + 1])[3] = (float)a;
  const int N = v.n_atoms;
  for (int q = 0; q < 4; q++) v.ej[(size_t)q * N + i] = 0;
  if (zero_first) {
    v.fx[i] = 0;
    v.fy[i] = 0;
    v.fz[i] = 0;
    v.gx[i] = 0.0;
    v.gy[i] = 0.0;
    v.gz[i] = 0.0;
    v.hx[i] = 0;
    v.hy[i] = 0;
    v.hz[i] = 0;
    if (i == v.atom_off[s])
      for (int k = 0; k < E_COUNT; k++)
        if (k != E_EKIN) v.ene[(size_t)s * E_COUNT + k] = 0.0;
  }
}

// --------------------------------------------------------------- K3 tiles
__global__ void __launch_bounds__(32 * kTileWarps, 5) k_gb_tile(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane & ~7, a = lane & 7;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sP[kTileWarps][8];
  __shared__ float red[kTileWarps][7][32];
  const int s = v.sc_sys[sc];
  const SysParams &P = v.sp[s];
  GbSettings gs;
  gs.load(P);
  const int a0 = v.sc_atom0[sc];
  const int end = v.atom_off[s + 1];
  const int na = min(32, end - a0);
  const int i = a0 + (lane < na ? lane : 0);
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ip = v.prm[i];
  float fx = 0.f, fy = 0.f, fz = 0.f, e_vdw = 0.f, e_el = 0.f, e_pol = 0.f, deda = 0.f;
  const int N = v.n_atoms;
  const int e1 = v.tile_e1[sc];
  int e = v.tile_e0[sc] + warp;
  JStage nx;
  if (e < e1) stage_load<1>(v, e, end, lane, nx);
  while (e < e1) {
    const JStage cur = nx;
    if (lane < cur.nb) {
      sA[warp][lane] = cur.a;
      sB[warp][lane] = cur.b;
      sP[warp][lane] = cur.c;
    }
    const unsigned rows = cur.row;
    unsigned xrows = 0, brows = 0;  // bond order <= 2, == 3
    if (cur.spec >= 0) {
      xrows = spec_row(v, cur.spec, 0, lane);
      brows = spec_row(v, cur.spec, 1, lane);
    }
    __syncwarp();
    const int en = e + kTileWarps;
    if (en < e1) stage_load<1>(v, en, end, lane, nx);
    float jacc[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
    for (int t = 0; t < 8; t++) {
      const int jt = (a + t) & 7;
      const float4 ja = sA[warp][jt], jb = sB[warp][jt], jp = sP[warp][jt];
      const Dx d = diff(ia, ib, ja, jb);
      const bool in = ((rows >> jt) & 1u) && d.r2 <= gs.rc2;
      float c[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (in) {
        const bool nb3 = !((xrows >> jt) & 1u);
        const bool b14 = (brows >> jt) & 1u;
        const GbPair gp = gb_pair_term(gs, d, nb3, b14, ib.w, jb.w, ia.w, ja.w, ip.x, jp.x, ip.y, jp.y, v, i,
                                       cur.b0 + jt);
        e_pol += gp.epol;
        deda += gp.dedal * jb.w;
        e_vdw += gp.vdw;
        e_el += gp.elec;
        fx -= gp.fscal * d.x;
        fy -= gp.fscal * d.y;
        fz -= gp.fscal * d.z;
        c[0] = gp.fscal * d.x;
        c[1] = gp.fscal * d.y;
        c[2] = gp.fscal * d.z;
        c[3] = gp.vdw;
        c[4] = gp.elec;
        c[5] = gp.epol;
        c[6] = gp.dedal * ib.w;
      }
      const int src = g8 | ((a - t) & 7);
#pragma unroll
      for (int q = 0; q < 7; q++) jacc[q] += __shfl_sync(0xffffffffu, c[q], src);
    }
#pragma unroll
    for (int q = 0; q < 7; q++) {
      jacc[q] += __shfl_xor_sync(0xffffffffu, jacc[q], 8);
      jacc[q] += __shfl_xor_sync(0xffffffffu, jacc[q], 16);
    }
    if (lane < cur.nb) {
      const int j = cur.b0 + lane;
      atomicAdd((unsigned long long *)&v.hx[j], (unsigned long long)to_fixed_j(jacc[0]));
      atomicAdd((unsigned long long *)&v.hy[j], (unsigned long long)to_fixed_j(jacc[1]));
      atomicAdd((unsigned long long *)&v.hz[j], (unsigned long long)to_fixed_j(jacc[2]));
#pragma unroll
      for (int q = 0; q < 4; q++)
        atomicAdd((unsigned long long *)&v.ej[(size_t)q * N + j], (unsigned long long)to_fixed_j(jacc[3 + q]));
    }
    __syncwarp();
    e = en;
  }
  // i side: the warps' partials in fixed order
  red[warp][0][lane] = fx;
  red[warp][1][lane] = fy;
  red[warp][2][lane] = fz;
  red[warp][3][lane] = e_vdw;
  red[warp][4][lane] = e_el;
  red[warp][5][lane] = e_pol;
  red[warp][6][lane] = deda;
  __syncthreads();
  if (warp == 0 && lane < na) {
    double t[7];
    for (int q = 0; q < 7; q++) {
      t[q] = 0.0;
      for (int w = 0; w < kTileWarps; w++) t[q] += (double)red[w][q][lane];
    }
    v.gx[i] += t[0];
    v.gy[i] += t[1];
    v.gz[i] += t[2];
    v.e_atom[(size_t)AE_VDW * N + i] = t[3];
    v.e_atom[(size_t)AE_ELEC * N + i] = t[4];
    v.e_atom[(size_t)AE_POL * N + i] = t[5];
    v.deda[i] = t[6];
  }
}

// Per-atom values of the fused pass from its i and j sides, as the row
// kernel leaves them: LJ and Coulomb halves, the GB pair sum, the self term,
// and the chain-rule weight gpi * dE/da_i (gbff.cpp:1731-1757).
__global__ void k_gb_finish(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  const int N = v.n_atoms;
  const SysParams &P = v.sp[v.sys_of[i]];
  double dv = v.e_atom[(size_t)AE_VDW * N + i] + (double)v.ej[i] * kInvJScale;
  double de = v.e_atom[(size_t)AE_ELEC * N + i] + (double)v.ej[(size_t)N + i] * kInvJScale;
  double dp = v.e_atom[(size_t)AE_POL * N + i] + (double)v.ej[(size_t)2 * N + i] * kInvJScale;
  double dd = v.deda[i] + (double)v.ej[(size_t)3 * N + i] * kInvJScale;
  double ai_d = v.born_d[i];
  double qd = (double)v.pq[2 * (size_t)i].w;
  double eself = P.premul_d * qd * qd / ai_d;
  v.e_atom[(size_t)AE_VDW * N + i] = 0.5 * dv;
  v.e_atom[(size_t)AE_ELEC * N + i] = 0.5 * de;
  v.e_atom[(size_t)AE_POL * N + i] = dp;
  v.e_atom[(size_t)AE_POL_SELF * N + i] = eself;
  double deda_i = dd - eself / ai_d;
  double gpi = ai_d * ai_d / 166.0;  // gbff.cpp:1755 uses the literal 166.0
  reinterpret_cast<float *>(&v.chainp[i])[2] = (float)(gpi * deda_i);
}

// --------------------------------------------------------------- K4 tiles
__global__ void __launch_bounds__(32 * kTileWarps) k_chain_tile(PackView v) {
  if (v.flags[F_NL_OVERFLOW]) return;
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane & ~7, a = lane & 7;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sC[kTileWarps][8];
  __shared__ float red[kTileWarps][3][32];
  const int s = v.sc_sys[sc];
  const SysParams &P = v.sp[s];
  const int a0 = v.sc_atom0[sc];
  const int end = v.atom_off[s + 1];
  const int na = min(32, end - a0);
  const int i = a0 + (lane < na ? lane : 0);
  const float4 ia = v.pq[2 * (size_t)i], ib = v.pq[2 * (size_t)i + 1], ic = v.chainp[i];
  const float s_hi = P.still2 * (1.f + 4e-6f), s_lo = P.still2 * (1.f - 4e-6f);
  const float invP5 = P.invP5, piP5 = P.piP5, P4 = P.P4;
  const double still2_d = P.still2_d;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  const int e1 = v.tile_e1[sc];
  int e = v.tile_e0[sc] + warp;
  JStage nx;
  if (e < e1) stage_load<0>(v, e, end, lane, nx);
  while (e < e1) {
    const JStage cur = nx;
    if (lane < cur.nb) {
      sA[warp][lane] = cur.a;
      sB[warp][lane] = cur.b;
      sC[warp][lane] = cur.c;
    }
    unsigned rows = cur.row;
    if (cur.spec >= 0) rows &= ~spec_row(v, cur.spec, 0, lane);  // bond order > 2 only
    __syncwarp();
    const int en = e + kTileWarps;
    if (en < e1) stage_load<0>(v, en, end, lane, nx);
    float j0 = 0.f, j1 = 0.f, j2 = 0.f;
#pragma unroll 2
    for (int t = 0; t < 8; t++) {
      const int jt = (a + t) & 7;
      float c0 = 0.f, c1 = 0.f, c2 = 0.f;
      if ((rows >> jt) & 1u) {
        const float4 ja = sA[warp][jt], jb = sB[warp][jt], jc = sC[warp][jt];
        const Dx d = diff(ia, ib, ja, jb);
        bool ok = d.r2 <= s_lo;
        if (!ok && d.r2 <= s_hi) {
          const int j = cur.b0 + jt;
          ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) > still2_d);
        }
        if (ok) {
          const float tt = chain_term(d, ic.x, jc.x, ic.y, jc.y, ic.z, jc.z, invP5, piP5, P4);
          fx += tt * d.x;
          fy += tt * d.y;
          fz += tt * d.z;
          c0 = -tt * d.x;
          c1 = -tt * d.y;
          c2 = -tt * d.z;
        }
      }
      const int src = g8 | ((a - t) & 7);
      j0 += __shfl_sync(0xffffffffu, c0, src);
      j1 += __shfl_sync(0xffffffffu, c1, src);
      j2 += __shfl_sync(0xffffffffu, c2, src);
    }
    j0 += __shfl_xor_sync(0xffffffffu, j0, 8);
    j1 += __shfl_xor_sync(0xffffffffu, j1, 8);
    j2 += __shfl_xor_sync(0xffffffffu, j2, 8);
    j0 += __shfl_xor_sync(0xffffffffu, j0, 16);
    j1 += __shfl_xor_sync(0xffffffffu, j1, 16);
    j2 += __shfl_xor_sync(0xffffffffu, j2, 16);
    if (lane < cur.nb) {
      const int j = cur.b0 + lane;
      atomicAdd((unsigned long long *)&v.hx[j], (unsigned long long)to_fixed_j(j0));
      atomicAdd((unsigned long long *)&v.hy[j], (unsigned long long)to_fixed_j(j1));
      atomicAdd((unsigned long long *)&v.hz[j], (unsigned long long)to_fixed_j(j2));
    }
    __syncwarp();
    e = en;
  }
  red[warp][0][lane] = fx;
  red[warp][1][lane] = fy;
  red[warp][2][lane] = fz;
  __syncthreads();
  if (warp == 0 && lane < na) {
    double t[3];
    for (int q = 0; q < 3; q++) {
      t[q] = 0.0;
      for (int w = 0; w < kTileWarps; w++) t[q] += (double)red[w][q][lane];
    }
    v.gx[i] += t[0];
    v.gy[i] += t[1];
    v.gz[i] += t[2];
  }
}

// instrumentation: out[0] += list pairs held by the tiles, out[1] += tiles
__global__ void k_tile_counts(PackView v, unsigned long long *out) {
  const int n = v.tile_count[0];
  unsigned long long p = 0, t = 0;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    for (int w = 0; w < 8; w++) p += __popc(v.tile_rows[8 * (size_t)e + w]);
    t++;
  }
  p = group_sum<32>(p);
  t = group_sum<32>(t);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], p);
    atomicAdd(&out[1], t);
  }
}
void launch_tile_counts(const PackView &v, cudaStream_t st, unsigned long long *out) {
  PDGPU_LAUNCH(k_tile_counts, 296, 256, 0, st, v, out);
}

// --------------------------------------------------------------- launchers
size_t tile_build_smem(int max_sys_atoms) {
  int nbits = (max_sys_atoms + 7) / 8;
  int W = (nbits + 31) / 32;
  return sizeof(unsigned) * (2 * (size_t)W + 1 + kBuildChunk + 3 * 8 * (size_t)kBuildChunk);
}
void launch_tiles_build(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  cudaMemsetAsync(v.tile_count, 0, 2 * sizeof(int), st);
  size_t smem = tile_build_smem(v.max_sys_atoms);
  static size_t opted = 0;  // dynamic shared memory above 48 KB needs an opt-in
  if (smem > 48 * 1024 && smem > opted) {
    cudaFuncSetAttribute(k_tile_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    opted = smem;
  }
  PDGPU_LAUNCH(k_tile_build, v.n_sc, 128, smem, st, v);
}
void launch_born_radii_tile(const PackView &v, cudaStream_t st, bool zero_first) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_born_tile, v.n_sc, 32 * kTileWarps, 0, st, v);
  PDGPU_LAUNCH(k_born_finish, (v.n_atoms + 63) / 64, 64, 0, st, v, (int)zero_first);
}
void launch_gb_pair_tile(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_gb_tile, v.n_sc, 32 * kTileWarps, 0, st, v);
  PDGPU_LAUNCH(k_gb_finish, (v.n_atoms + 63) / 64, 64, 0, st, v);
}
void launch_gb_chain_tile(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH(k_chain_tile, v.n_sc, 32 * kTileWarps, 0, st, v);
}

}  // namespace pdgpu
