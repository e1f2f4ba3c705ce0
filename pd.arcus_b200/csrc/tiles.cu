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
// Each pass runs a persistent grid of G warps over the pack's T tiles
// (every system's clusters, the tiles of a cluster consecutive): warp g
// takes the contiguous range [T g / G, T (g+1) / G), so every warp gets the
// same number of tiles, give or take one, however unequal the clusters'
// tile counts are.  A warp prefetches the next tile's 8 j atoms while it
// works on the current one, and reloads its i atoms when the range enters
// the next cluster.  Lane l = 8g + a (one i atom) walks the tile's j atoms
// in the order (a+t) mod 8: the i side accumulates in registers, the j
// side goes with one shuffle to the lane of its group that owns the j
// atom; after the 8 steps the four groups' j sums meet with two xor
// shuffles.  Both sides of each tile are then added to their atoms with
// 64-bit fixed-point atomics.  A tile's sums depend on the tile alone, and
// fixed-point sums do not depend on the order of the additions, so every
// result is bit-identical run to run, however the tiles are spread over
// the warps and whatever other systems share the pack.  Pass results:
//   K2 k_born_tile   Born sums, fixed point 2^40 (exact per term);
//                    k_born_finish inverts them (FP64) and zeroes the
//                    accumulators of the next passes
//   K3 k_gb_tile     forces, per-atom LJ / Coulomb / GB energies and dE/da,
//                    fixed point 2^24; k_gb_finish forms the reference's
//                    per-atom values and the chain-rule weights
//   K4 k_chain_tile  chain-rule forces, fixed point 2^24
// The per-pair arithmetic is the row kernels' (pairmath.cuh).
#include <cuda_runtime.h>

#include <algorithm>

#include "tilecommon.cuh"

namespace pdgpu {

constexpr int kTileWarps = 4;    // warps per block
// resident blocks per SM the register allocation must allow, per pass
#ifndef PDGPU_K2_BLOCKS
#define PDGPU_K2_BLOCKS 6
#endif
#ifndef PDGPU_K3_BLOCKS
#define PDGPU_K3_BLOCKS 5
#endif
#ifndef PDGPU_K4_BLOCKS
#define PDGPU_K4_BLOCKS 6
#endif
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
      const int nb = min(8, end - cb0[r]);
      v.tile_meta[et] = make_int4(cb0[r], spec, a0, (s << 8) | ((na - 1) << 3) | (nb - 1));
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------- tile search
// The tiles straight from the positions, without the list.  The pair test
// is the list's (the reference's FP64 expression without contraction,
// neighbourlist.cpp:263-266, and j != i) and the bond orders come from the
// same band and off-diagonal tables, so the tiles hold exactly the pairs a
// list build at these positions would give them.
//
// (1) k_cluster_boxes: one thread per j-cluster folds its <= 8 atoms into
// an FP64 box (a cluster with a NaN coordinate gets an infinite box: its
// pairs are decided by the distance test alone) and saves the positions of
// this rebuild (for a later list build at the same positions).
// (2) k_tile_search: one block per i-cluster; its warps take the system's
// j-clusters at or after the i-cluster 32 at a time, one per lane, and keep
// those whose box lies within the list cutoff of the i-cluster's box (a
// margin of 1e-9 relative keeps the cull conservative); for each kept
// j-cluster the warp tests its 32 x 8 atom pairs (lane = i atom) and emits
// a tile when any pair is in.
__global__ void k_cluster_boxes(PackView v) {
  const int jc = blockIdx.x * blockDim.x + threadIdx.x;
  if (jc >= v.n_jc) return;
  const int a0 = v.jc_atom0[jc];
  const int s = v.sys_of[a0];
  const int n = min(8, v.atom_off[s + 1] - a0);
  const int N = v.n_atoms;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool wild = false;
  for (int k = 0; k < n; k++) {
    const int i = a0 + k;
    const double p[3] = {v.x[i], v.y[i], v.z[i]};
    for (int c = 0; c < 3; c++) {
      wild |= !(p[c] == p[c]);
      lo[c] = fmin(lo[c], p[c]);
      hi[c] = fmax(hi[c], p[c]);
      v.xs[(size_t)c * N + i] = p[c];
    }
  }
  for (int c = 0; c < 3; c++) {
    v.cbox[6 * (size_t)jc + c] = wild ? -INFINITY : lo[c];
    v.cbox[6 * (size_t)jc + 3 + c] = wild ? INFINITY : hi[c];
  }
}

constexpr int kSearchWarps = 8;  // warps per i-cluster block of the tile search

// One candidate j-cluster against this lane's i atom: the pair bits and
// the bond-order bits (<= 2, == 3).  The pair tests come first (the 8 j
// positions load independently), then the bond orders of the pairs in
// (independent band loads).
struct SearchRow {
  unsigned row, xr, br;
};
__device__ __forceinline__ SearchRow search_row(const PackView &v, bool live, int i, int li, int a0, double xi,
                                                double yi, double zi, double lim, int jb0, int nb, int o,
                                                int mid, const signed char *band, bool has_off, int s) {
  SearchRow r = {0u, 0u, 0u};
  if (!live) return r;
#pragma unroll
  for (int t = 0; t < 8; t++) {
    const int j = jb0 + t;
    // the half list: j > i inside the i-cluster
    if (t < nb && !(j <= i && j < a0 + 32) && !(ref_d2(xi, yi, zi, v.x[j], v.y[j], v.z[j]) > lim))
      r.row |= 1u << t;
  }
#pragma unroll
  for (int t = 0; t < 8; t++) {
    if (!((r.row >> t) & 1u)) continue;
    const int lj = jb0 + t - o;
    const int delta = lj > li ? lj - li : li - lj;
    int bo = 7;
    if (delta < mid)
      bo = band[(long long)min(li, lj) * mid + (delta - 1)];
    else if (has_off)
      bo = bond_order(v, s, i, jb0 + t);
    if (bo <= 2)
      r.xr |= 1u << t;
    else if (bo == 3)
      r.br |= 1u << t;
  }
  return r;
}
// A search block's tiles are staged in shared memory and written to the
// tile store as one contiguous range by the block's last warp to finish, so
// the tiles of an i-cluster sit together and a pass that walks contiguous
// tile ranges meets few i-cluster changes (each one a reload of the i side).
// Tiles beyond the staging capacity go to the store one at a time.
constexpr int kSearchStage = 256;
struct SearchStage {
  int n;                               // tiles emitted into the stage (may pass kSearchStage)
  int done;                            // warps that have finished their j-clusters
  int4 meta[kSearchStage];
  unsigned rows[kSearchStage * 8];     // byte l of tile k's 32 bytes = i lane l's bits
};
// Store one tile (when any pair is in); false when a capacity ran out
// (cannot happen: the capacities are worst cases).
__device__ __forceinline__ bool search_emit(const PackView &v, int lane, const SearchRow &r, int jb0, int a0, int s,
                                            int na, int nb, SearchStage &stage) {
  if (!__any_sync(0xffffffffu, r.row != 0)) return true;
  int spec = -1;
  if (__any_sync(0xffffffffu, (r.xr | r.br) != 0)) {
    if (lane == 0) spec = atomicAdd(&v.tile_count[1], 1);
    spec = __shfl_sync(0xffffffffu, spec, 0);
    if (spec >= v.spec_cap) {
      if (lane == 0) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
      return false;
    }
    reinterpret_cast<unsigned char *>(v.spec_rows)[64 * (size_t)spec + lane] = (unsigned char)r.xr;
    reinterpret_cast<unsigned char *>(v.spec_rows)[64 * (size_t)spec + 32 + lane] = (unsigned char)r.br;
  }
  const int4 meta = make_int4(jb0, spec, a0, (s << 8) | ((na - 1) << 3) | (nb - 1));
  int k = 0;
  if (lane == 0) k = atomicAdd(&stage.n, 1);
  k = __shfl_sync(0xffffffffu, k, 0);
  if (k < kSearchStage) {
    reinterpret_cast<unsigned char *>(stage.rows)[32 * k + lane] = (unsigned char)r.row;
    if (lane == 0) stage.meta[k] = meta;
    return true;
  }
  int e = 0;
  if (lane == 0) e = atomicAdd(&v.tile_count[0], 1);
  e = __shfl_sync(0xffffffffu, e, 0);
  if (e >= v.tile_cap) {
    if (lane == 0) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
    return false;
  }
  reinterpret_cast<unsigned char *>(v.tile_rows)[32 * (size_t)e + lane] = (unsigned char)r.row;
  if (lane == 0) v.tile_meta[e] = meta;
  return true;
}

__global__ void __launch_bounds__(32 * kSearchWarps, 5) k_tile_search(PackView v) {
  const int sc = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = v.sc_sys[sc];
  const int a0 = v.sc_atom0[sc];
  const int end = v.atom_off[s + 1];
  const int na = min(32, end - a0);
  const int jc0 = v.sc_jc0[sc], jc_end = v.jc_off[s + 1];
  const double lim = v.sp[s].nl_lim2_d;
  const double cull = lim * (1.0 + 1e-9);
  // the i-cluster's box: its (up to four) j-clusters' boxes
  double ilo[3] = {INFINITY, INFINITY, INFINITY}, ihi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int q = 0; q < 4 && jc0 + q < jc_end; q++)
    for (int c = 0; c < 3; c++) {
      ilo[c] = fmin(ilo[c], v.cbox[6 * (size_t)(jc0 + q) + c]);
      ihi[c] = fmax(ihi[c], v.cbox[6 * (size_t)(jc0 + q) + 3 + c]);
    }
  // this lane's i atom and what its bond orders need
  const bool live = lane < na;
  const int i = a0 + (live ? lane : 0);
  const double xi = v.x[i], yi = v.y[i], zi = v.z[i];
  const int o = v.atom_off[s], mid = v.mid[s], li = i - o;
  const signed char *band = reinterpret_cast<const signed char *>(v.band) + v.band_off[s];
  const bool has_off = v.off_ptr[i + 1] > v.off_ptr[i];
  // the i atoms' positions for the per-atom cull
  __shared__ double sx[32], sy[32], sz[32];
  __shared__ SearchStage stage;
  __shared__ int stop_s;  // an earlier overflow, read once so every thread of the block agrees
  if (threadIdx.x == 0) {
    stage.n = 0;
    stage.done = 0;
    stop_s = v.flags[F_NL_OVERFLOW];
  }
  if (warp == 0) {
    sx[lane] = xi;
    sy[lane] = yi;
    sz[lane] = zi;
  }
  __syncthreads();
  if (stop_s) return;
  bool ok = true;  // false once a capacity ran out (warp-uniform)
  for (int base = jc0 + 32 * warp; ok && base < jc_end; base += 32 * kSearchWarps) {
    bool cand = false;
    const int jc = base + lane;
    if (jc < jc_end) {
      double jlo[3], jhi[3];
      for (int c = 0; c < 3; c++) {
        jlo[c] = v.cbox[6 * (size_t)jc + c];
        jhi[c] = v.cbox[6 * (size_t)jc + 3 + c];
      }
      double g2 = 0.0;
      for (int c = 0; c < 3; c++) {
        const double gap = fmax(0.0, fmax(jlo[c] - ihi[c], ilo[c] - jhi[c]));
        g2 += gap * gap;
      }
      cand = !(g2 > cull);  // NaN (infinite boxes): a candidate
      // boxes this close: some i atom must lie within the cutoff of the
      // j-cluster's box (an i-cluster across two chains has a large box)
      if (cand) {
        cand = false;
        for (int k = 0; k < na && !cand; k++) {
          const double p[3] = {sx[k], sy[k], sz[k]};
          double h2 = 0.0;
          for (int c = 0; c < 3; c++) {
            const double gap = fmax(0.0, fmax(jlo[c] - p[c], p[c] - jhi[c]));
            h2 += gap * gap;
          }
          cand = !(h2 > cull);
        }
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, cand);
    // two candidates at a time: their loads overlap
    while (ok && m) {
      const int q1 = __ffs(m) - 1;
      m &= m - 1;
      const int q2 = m ? __ffs(m) - 1 : -1;
      if (m) m &= m - 1;
      const int jb1 = v.jc_atom0[base + q1], nb1 = min(8, end - jb1);
      const int jb2 = q2 >= 0 ? v.jc_atom0[base + q2] : jb1, nb2 = min(8, end - jb2);
      const SearchRow r1 = search_row(v, live, i, li, a0, xi, yi, zi, lim, jb1, nb1, o, mid, band, has_off, s);
      SearchRow r2 = {0u, 0u, 0u};
      if (q2 >= 0) r2 = search_row(v, live, i, li, a0, xi, yi, zi, lim, jb2, nb2, o, mid, band, has_off, s);
      ok = search_emit(v, lane, r1, jb1, a0, s, na, nb1, stage);
      if (ok && q2 >= 0) ok = search_emit(v, lane, r2, jb2, a0, s, na, nb2, stage);
    }
  }
  // the staged tiles as one range of the tile store, written by the last
  // warp to finish; the others exit at once (a warp with no j-clusters does
  // not hold its slot while the block's busy warps run)
  __syncwarp();
  __threadfence_block();  // this warp's stage writes before its count
  int last = 0;
  if (lane == 0) last = atomicAdd(&stage.done, 1) == kSearchWarps - 1;
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __syncwarp();
  __threadfence_block();  // every warp's stage writes after the count
  const int n = min(*(volatile int *)&stage.n, kSearchStage);
  if (n == 0) return;
  long long b0 = 0;
  if (lane == 0) b0 = atomicAdd(&v.tile_count[0], n);
  b0 = __shfl_sync(0xffffffffu, b0, 0);
  if (b0 + n > v.tile_cap) {
    if (lane == 0) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
    return;
  }
  const volatile unsigned *rows = stage.rows;
  for (int w = lane; w < 8 * n; w += 32) v.tile_rows[8 * b0 + w] = rows[w];
  for (int k = lane; k < n; k += 32) {
    const volatile int *m = reinterpret_cast<const volatile int *>(&stage.meta[k]);
    v.tile_meta[b0 + k] = make_int4(m[0], m[1], m[2], m[3]);
  }
}

// --------------------------------------------------------------- tile passes
// Staging of a tile: its metadata and this lane's row bits, and in lanes
// 0..7 three records of their j atom, held in registers (prefetched one
// tile ahead) and written to the warp's shared slots before the tile is
// processed.
struct JStage {
  float4 a, b, c;
  int4 m;
  unsigned row;
};
template <int REC>  // third record: 0 chainp (radius R, volume V, chain weight w), 1 prm (LJ radius, eps)
__device__ __forceinline__ void stage_load(const PackView &v, int e, int lane, JStage &q) {
  q.m = v.tile_meta[e];
  q.row = tile_row(v, e, lane);
  if (lane <= (q.m.w & 7)) {
    const int j = q.m.x + lane;
    q.a = v.pq[2 * (size_t)j];
    q.b = v.pq[2 * (size_t)j + 1];
    q.c = REC == 0 ? v.chainp[j] : v.prm[j];
  }
}

// This warp's tile range [e0, e1): an equal share of the pack's tiles.
__device__ __forceinline__ void warp_range(const PackView &v, int warp, int &e0, int &e1) {
  const long long T = v.tile_count[0];
  const long long G = (long long)gridDim.x * kTileWarps;
  const long long g = (long long)blockIdx.x * kTileWarps + warp;
  e0 = (int)(T * g / G);
  e1 = (int)(T * (g + 1) / G);
}

// --------------------------------------------------------------- K2 tiles
// (register bounds: five blocks per SM)
__global__ void __launch_bounds__(32 * kTileWarps, PDGPU_K2_BLOCKS) k_born_tile(PackView v) {
  PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane & ~7, a = lane & 7;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sC[kTileWarps][8];
  int e, e1;
  warp_range(v, warp, e, e1);
  if (e >= e1) return;
  JStage nx;
  stage_load<0>(v, e, lane, nx);
  int a0 = -1, na = 0, i = 0;
  float4 ia, ib, ic;
  float s_hi = 0.f, s_lo = 0.f, invP5 = 0.f, piP5 = 0.f, P4s = 0.f;
  double still2_d = 0.0;
  long long acc_i = 0;  // exact per term: added when the range leaves the cluster
  for (; e < e1; e++) {
    const JStage cur = nx;
    const TileInfo ti = tile_info(cur.m);
    if (e + 1 < e1) stage_load<0>(v, e + 1, lane, nx);
    if (ti.a0 != a0) {
      if (lane < na && acc_i) atomicAdd((unsigned long long *)&v.bsum[a0 + lane], (unsigned long long)acc_i);
      acc_i = 0;
      a0 = ti.a0;
      na = ti.na;
      i = a0 + (lane < na ? lane : 0);
      ia = v.pq[2 * (size_t)i];
      ib = v.pq[2 * (size_t)i + 1];
      ic = v.chainp[i];
      const SysParams &P = v.sp[ti.s];
      s_hi = P.still2 * (1.f + 4e-6f);
      s_lo = P.still2 * (1.f - 4e-6f);
      invP5 = P.invP5;
      piP5 = P.piP5;
      P4s = P.P4 * (float)kBornScale;
      still2_d = P.still2_d;
    }
    if (lane < ti.nb) {
      sA[warp][lane] = cur.a;
      sB[warp][lane] = cur.b;
      sC[warp][lane] = cur.c;
    }
    unsigned rows = cur.row;
    if (ti.spec >= 0) rows &= ~spec_row(v, ti.spec, 0, lane);  // bond order > 2 only
    __syncwarp();
    long long jacc = 0;  // lane (g,a): j atom a, this group's i atoms
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const int jt = (a + t) & 7;
      long long tI = 0, tJ = 0;
      if ((rows >> jt) & 1u) {
        const float4 ja = sA[warp][jt], jb = sB[warp][jt], jc = sC[warp][jt];
        const Dx d = diff(ia, ib, ja, jb);
        bool ok = d.r2 <= s_lo;
        if (!ok && d.r2 <= s_hi) {
          const int j = ti.b0 + jt;
          ok = !(ref_d2(v.x[i], v.y[i], v.z[i], v.x[j], v.y[j], v.z[j]) > still2_d);
        }
        if (ok) {
          const float term = born_term_noV(d, ic.x, jc.x, invP5, piP5, P4s);
          tI = __float2ll_rn(__fmul_rn(term, jc.y));
          tJ = __float2ll_rn(__fmul_rn(term, ic.y));
        }
      }
      acc_i += tI;
      jacc += __shfl_sync(0xffffffffu, tJ, g8 | ((a - t) & 7));
    }
    jacc += __shfl_xor_sync(0xffffffffu, jacc, 8);
    jacc += __shfl_xor_sync(0xffffffffu, jacc, 16);
    if (lane < ti.nb && jacc) atomicAdd((unsigned long long *)&v.bsum[ti.b0 + lane], (unsigned long long)jacc);
    __syncwarp();
  }
  if (lane < na && acc_i) atomicAdd((unsigned long long *)&v.bsum[a0 + lane], (unsigned long long)acc_i);
}

// a_i = -halfeconv / (terms123_i + sum) (FP64); zero the accumulators the
// following passes add into (and, first in an evaluation, the forces)
__global__ void k_born_finish(PackView v, int zero_first) {
  PDGPU_DEP_ENTRY();
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
    if (zero_first & ZF_BONDED) {
      v.fx[i] = 0;
      v.fy[i] = 0;
      v.fz[i] = 0;
    }
    v.gx[i] = 0.0;
    v.gy[i] = 0.0;
    v.gz[i] = 0.0;
    v.hx[i] = 0;
    v.hy[i] = 0;
    v.hz[i] = 0;
    if ((zero_first & ZF_RECORD) && i == v.atom_off[s]) {
      for (int k = 0; k < E_COUNT; k++)
        if (k != E_EKIN) v.ene[(size_t)s * E_COUNT + k] = 0.0;
      v.sys_flags[s] = 0;
    }
  }
}

// --------------------------------------------------------------- K3 tiles
__global__ void __launch_bounds__(32 * kTileWarps, PDGPU_K3_BLOCKS) k_gb_tile(PackView v) {
  PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane & ~7, a = lane & 7;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sP[kTileWarps][8];
  int e, e1;
  warp_range(v, warp, e, e1);
  if (e >= e1) return;
  const int N = v.n_atoms;
  JStage nx;
  stage_load<1>(v, e, lane, nx);
  int a0 = -1, i = 0;
  float4 ia, ib, ip;
  GbSettings gs;
  for (; e < e1; e++) {
    const JStage cur = nx;
    const TileInfo ti = tile_info(cur.m);
    if (e + 1 < e1) stage_load<1>(v, e + 1, lane, nx);
    if (ti.a0 != a0) {
      a0 = ti.a0;
      i = a0 + (lane < ti.na ? lane : 0);
      ia = v.pq[2 * (size_t)i];
      ib = v.pq[2 * (size_t)i + 1];
      ip = v.prm[i];
      gs.load(v.sp[ti.s]);
    }
    if (lane < ti.nb) {
      sA[warp][lane] = cur.a;
      sB[warp][lane] = cur.b;
      sP[warp][lane] = cur.c;
    }
    const unsigned rows = cur.row;
    unsigned xrows = 0, brows = 0;  // bond order <= 2, == 3
    if (ti.spec >= 0) {
      xrows = spec_row(v, ti.spec, 0, lane);
      brows = spec_row(v, ti.spec, 1, lane);
    }
    __syncwarp();
    float fx = 0.f, fy = 0.f, fz = 0.f, e_vdw = 0.f, e_el = 0.f, e_pol = 0.f, deda = 0.f;
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
                                       ti.b0 + jt);
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
    if (lane < ti.nb) {
      const int j = ti.b0 + lane;
      add_fixed(v, &v.hx[j], jacc[0], ti.s);
      add_fixed(v, &v.hy[j], jacc[1], ti.s);
      add_fixed(v, &v.hz[j], jacc[2], ti.s);
#pragma unroll
      for (int q = 0; q < 4; q++) add_fixed(v, &v.ej[(size_t)q * N + j], jacc[3 + q], ti.s);
    }
    if (lane < ti.na) {
      add_fixed(v, &v.hx[i], fx, ti.s);
      add_fixed(v, &v.hy[i], fy, ti.s);
      add_fixed(v, &v.hz[i], fz, ti.s);
      add_fixed(v, &v.ej[i], e_vdw, ti.s);
      add_fixed(v, &v.ej[(size_t)N + i], e_el, ti.s);
      add_fixed(v, &v.ej[(size_t)2 * N + i], e_pol, ti.s);
      add_fixed(v, &v.ej[(size_t)3 * N + i], deda, ti.s);
    }
    __syncwarp();
  }
}

// Per-atom values of the fused pass, as the row kernel leaves them: LJ and
// Coulomb halves, the GB pair sum, the self term, and the chain-rule
// weight gpi * dE/da_i (gbff.cpp:1731-1757).
__global__ void k_gb_finish(PackView v) {
  PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  const int N = v.n_atoms;
  const SysParams &P = v.sp[v.sys_of[i]];
  double dv = (double)v.ej[i] * kInvJScale;
  double de = (double)v.ej[(size_t)N + i] * kInvJScale;
  double dp = (double)v.ej[(size_t)2 * N + i] * kInvJScale;
  double dd = (double)v.ej[(size_t)3 * N + i] * kInvJScale;
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
__global__ void __launch_bounds__(32 * kTileWarps, PDGPU_K4_BLOCKS) k_chain_tile(PackView v) {
  PDGPU_DEP_ENTRY();
  if (v.flags[F_NL_OVERFLOW]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g8 = lane & ~7, a = lane & 7;
  __shared__ float4 sA[kTileWarps][8], sB[kTileWarps][8], sC[kTileWarps][8];
  int e, e1;
  warp_range(v, warp, e, e1);
  if (e >= e1) return;
  JStage nx;
  stage_load<0>(v, e, lane, nx);
  int a0 = -1, i = 0;
  float4 ia, ib, ic;
  float s_hi = 0.f, s_lo = 0.f, invP5 = 0.f, piP5 = 0.f, P4 = 0.f;
  double still2_d = 0.0;
  for (; e < e1; e++) {
    const JStage cur = nx;
    const TileInfo ti = tile_info(cur.m);
    if (e + 1 < e1) stage_load<0>(v, e + 1, lane, nx);
    if (ti.a0 != a0) {
      a0 = ti.a0;
      i = a0 + (lane < ti.na ? lane : 0);
      ia = v.pq[2 * (size_t)i];
      ib = v.pq[2 * (size_t)i + 1];
      ic = v.chainp[i];
      const SysParams &P = v.sp[ti.s];
      s_hi = P.still2 * (1.f + 4e-6f);
      s_lo = P.still2 * (1.f - 4e-6f);
      invP5 = P.invP5;
      piP5 = P.piP5;
      P4 = P.P4;
      still2_d = P.still2_d;
    }
    if (lane < ti.nb) {
      sA[warp][lane] = cur.a;
      sB[warp][lane] = cur.b;
      sC[warp][lane] = cur.c;
    }
    unsigned rows = cur.row;
    if (ti.spec >= 0) rows &= ~spec_row(v, ti.spec, 0, lane);  // bond order > 2 only
    __syncwarp();
    float fx = 0.f, fy = 0.f, fz = 0.f, j0 = 0.f, j1 = 0.f, j2 = 0.f;
#pragma unroll 2
    for (int t = 0; t < 8; t++) {
      const int jt = (a + t) & 7;
      float c0 = 0.f, c1 = 0.f, c2 = 0.f;
      if ((rows >> jt) & 1u) {
        const float4 ja = sA[warp][jt], jb = sB[warp][jt], jc = sC[warp][jt];
        const Dx d = diff(ia, ib, ja, jb);
        bool ok = d.r2 <= s_lo;
        if (!ok && d.r2 <= s_hi) {
          const int j = ti.b0 + jt;
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
    if (lane < ti.nb) {
      const int j = ti.b0 + lane;
      add_fixed(v, &v.hx[j], j0, ti.s);
      add_fixed(v, &v.hy[j], j1, ti.s);
      add_fixed(v, &v.hz[j], j2, ti.s);
    }
    if (lane < ti.na) {
      add_fixed(v, &v.hx[i], fx, ti.s);
      add_fixed(v, &v.hy[i], fy, ti.s);
      add_fixed(v, &v.hz[i], fz, ti.s);
    }
    __syncwarp();
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
// Persistent grids: the blocks one wave holds, and no more warps than the
// pack can have tiles.
void tile_launch_shapes(PackView &v) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int occ[3] = {1, 1, 1};
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_born_tile, 32 * kTileWarps, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_gb_tile, 32 * kTileWarps, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], k_chain_tile, 32 * kTileWarps, 0);
  const long long need = (v.tile_cap + kTileWarps - 1) / kTileWarps;
  for (int p = 0; p < 3; p++)
    v.tile_blocks[p] = (int)std::max(1LL, std::min((long long)std::max(occ[p], 1) * sms, need));
  v.ev_blocks = eval_tiles_grid(v.tile_cap);
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
void launch_tiles_search(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  cudaMemsetAsync(v.tile_count, 0, 2 * sizeof(int), st);
  PDGPU_LAUNCH(k_cluster_boxes, (v.n_jc + 127) / 128, 128, 0, st, v);
  PDGPU_LAUNCH(k_tile_search, v.n_sc, 32 * kSearchWarps, 0, st, v);
}
void launch_born_radii_tile(const PackView &v, cudaStream_t st, int zero_first) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH_DEP(k_born_tile, v.tile_blocks[0], 32 * kTileWarps, 0, st, v);
  PDGPU_LAUNCH_DEP(k_born_finish, (v.n_atoms + 63) / 64, 64, 0, st, v, zero_first);
}
void launch_gb_pair_tile(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH_DEP(k_gb_tile, v.tile_blocks[1], 32 * kTileWarps, 0, st, v);
  PDGPU_LAUNCH_DEP(k_gb_finish, (v.n_atoms + 63) / 64, 64, 0, st, v);
}
void launch_gb_chain_tile(const PackView &v, cudaStream_t st) {
  if (!v.n_sc) return;
  PDGPU_LAUNCH_DEP(k_chain_tile, v.tile_blocks[2], 32 * kTileWarps, 0, st, v);
}

}  // namespace pdgpu
