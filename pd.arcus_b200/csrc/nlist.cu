// K1: neighbour-list rebuild.
//
// Reference: NeighbourList::calcNewList_InfiniteSpace and
// correctOffDiagonalBondOrders (workspace/neighbourlist.cpp:162-316), an
// O(N^2) double loop.  Here: per-system cell grid (cell edge >= list
// cutoff) -> integer cell keys -> stable LSD radix sort (8-bit digits,
// warp-multisplit ranking) -> cell ranges -> warp-per-atom scan of the 27
// neighbouring cells.  The pair test is the reference's FP64 expression
// evaluated without contraction, (dx*dx + dy*dy) + dz*dz > (Rc+pad)^2, so the
// pair set is bit-identical.  Two passes (count, fill) give an exact CSR.
// Rows hold (j_global << 3) | bondorder; row order is the cell-scan order
// (the export sorts rows to the reference's ascending order).
//
// Roofline: HBM-bound integer/FP64 work.  Algorithmic bytes per rebuild:
// 36 B/atom (FP64 position read, key, index, offset) + 4 B per list entry.
#include <cuda_runtime.h>

#include "internal.cuh"

namespace pdgpu {

// --------------------------------------------------------------- grid plan
// Bounding boxes: every atom folds its coordinates into its system's box
// with 64-bit atomic min/max on an order-preserving integer image of the
// double (one warp-reduced atomic per warp when the warp lies in one
// system).  NaN coordinates are ignored for the box (their pairs are
// decided by the distance test alone, as in the reference).
__device__ __forceinline__ unsigned long long ordered_key(double d) {
  unsigned long long u = (unsigned long long)__double_as_longlong(d);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __forceinline__ double ordered_value(unsigned long long k) {
  unsigned long long u = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  return __longlong_as_double((long long)u);
}

__global__ void k_bbox(PackView v) {
  const int lane = threadIdx.x & 31;
  const int S = v.n_sys;
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < v.n_atoms;
       base += gridDim.x * blockDim.x) {
    int i = base + lane;
    bool valid = i < v.n_atoms;
    int s = valid ? v.sys_of[i] : -1;
    double p[3] = {valid ? v.x[i] : 0.0, valid ? v.y[i] : 0.0, valid ? v.z[i] : 0.0};
    double mn[3], mx[3];
    for (int k = 0; k < 3; k++) {
      bool ok = valid && p[k] == p[k];
      mn[k] = ok ? p[k] : 1e308;
      mx[k] = ok ? p[k] : -1e308;
    }
    int s0 = __shfl_sync(0xffffffffu, s, 0);
    bool uniform = __all_sync(0xffffffffu, s == s0 || s < 0);
    if (uniform) {
      for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 3; k++) {
          mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
          mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
      if (lane == 0 && s0 >= 0)
        for (int k = 0; k < 3; k++) {
          if (mn[k] <= mx[k]) {
            atomicMin(&v.bbox[k * S + s0], ordered_key(mn[k]));
            atomicMax(&v.bbox[(3 + k) * S + s0], ordered_key(mx[k]));
          }
        }
    } else if (s >= 0) {
      for (int k = 0; k < 3; k++)
        if (mn[k] <= mx[k]) {
          atomicMin(&v.bbox[k * S + s], ordered_key(mn[k]));
          atomicMax(&v.bbox[(3 + k) * S + s], ordered_key(mx[k]));
        }
    }
  }
}

// One thread per system: cell size and dims from the box.  Cells per system
// are capped at 2*natoms+64 (the key space is allocated from atom_off); a
// sparse system gets larger cells, which is still exact (more candidates
// only).
__global__ void k_grid_plan(PackView v) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= v.n_sys) return;
  const int S = v.n_sys;
  int a0 = v.atom_off[s], a1 = v.atom_off[s + 1];
  {
    double lo[3], ext[3];
    for (int k = 0; k < 3; k++) {
      lo[k] = ordered_value(v.bbox[k * S + s]);
      double hi = ordered_value(v.bbox[(3 + k) * S + s]);
      if (!(hi >= lo[k])) {  // empty or all-NaN system
        lo[k] = 0;
        hi = 0;
      }
      ext[k] = hi - lo[k];
    }
    double cell = sqrt(v.sp[s].nl_lim2_d) * (1.0 + 1e-12);
    double cap = 2.0 * (a1 - a0) + 64.0;
    // dimensions in double so huge or infinite extents cannot overflow; a
    // single cell is always exact (every pair is distance-tested)
    double fx = 1, fy = 1, fz = 1;
    bool ok = false;
    bool finite = ext[0] < 1e15 && ext[1] < 1e15 && ext[2] < 1e15;
    for (int it = 0; finite && it < 64; it++) {
      fx = floor(ext[0] / cell) + 1;
      fy = floor(ext[1] / cell) + 1;
      fz = floor(ext[2] / cell) + 1;
      if (fx * fy * fz <= cap) {
        ok = true;
        break;
      }
      if (it == 0) atomicExch(&v.flags[F_CELL_CLAMP], 1);
      cell *= 1.25;
    }
    if (!ok) {
      fx = fy = fz = 1;
      cell = 1e300;
      for (int k = 0; k < 3; k++) lo[k] = 0;
    }
    long long nx = (long long)fx, ny = (long long)fy, nz = (long long)fz;
    double *g = v.grid + 8 * s;
    g[0] = lo[0];
    g[1] = lo[1];
    g[2] = lo[2];
    g[3] = cell;
    g[4] = (double)nx;
    g[5] = (double)ny;
    g[6] = (double)nz;
    g[7] = (double)(2LL * a0 + 64LL * s);  // cell-key offset of this system
  }
}

__device__ __forceinline__ void cell_of(const double *g, double x, double y, double z, int &cx, int &cy,
                                        int &cz) {
  int nx = (int)g[4], ny = (int)g[5], nz = (int)g[6];
  double inv = 1.0 / g[3];
  double fx = (x - g[0]) * inv, fy = (y - g[1]) * inv, fz = (z - g[2]) * inv;
  // NaN, infinite or out-of-box coordinates clamp into the grid (fmax of a
  // NaN returns the other operand); the exact distance test still decides
  // every pair.
  cx = (int)fmin(fmax(fx, 0.0), (double)(nx - 1));
  cy = (int)fmin(fmax(fy, 0.0), (double)(ny - 1));
  cz = (int)fmin(fmax(fz, 0.0), (double)(nz - 1));
}

__global__ void k_cell_keys(PackView v, int *keys, int *vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_atoms) return;
  int s = v.sys_of[i];
  const double *g = v.grid + 8 * s;
  int cx, cy, cz;
  cell_of(g, v.x[i], v.y[i], v.z[i], cx, cy, cz);
  int nx = (int)g[4], ny = (int)g[5];
  keys[i] = (int)g[7] + (cz * ny + cy) * nx + cx;
  vals[i] = i;
}

// --------------------------------------------------------------- radix sort
// Stable LSD radix sort of (key, value) pairs, 8-bit digits, tiles of 2048.
constexpr int kTile = 2048;
constexpr int kSortThreads = 256;

__global__ void k_radix_hist(const int *keys, int n, int shift, int *hist, int ntiles) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kTile;
  for (int k = threadIdx.x; k < kTile; k += kSortThreads) {
    int idx = base + k;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & 255], 1);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of a small int array in one block (len up to a few 1e5)
__global__ void k_scan_small(int *a, int len) {
  __shared__ int part[1024];
  int t = threadIdx.x;
  int per = (len + blockDim.x - 1) / blockDim.x;
  int b = t * per, e = min(b + per, len);
  int s = 0;
  for (int k = b; k < e; k++) s += a[k];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < blockDim.x; off <<= 1) {
    int val = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += val;
    __syncthreads();
  }
  int run = part[t] - s;
  for (int k = b; k < e; k++) {
    int x = a[k];
    a[k] = run;
    run += x;
  }
}

__global__ void k_radix_scatter(const int *keys_in, const int *vals_in, int *keys_out, int *vals_out,
                                int n, int shift, const int *hist, int ntiles) {
  __shared__ int running[256];
  __shared__ int wcount[kSortThreads / 32][256];
  __shared__ int goff[256];
  int t = threadIdx.x, w = t >> 5, lane = t & 31;
  running[t] = 0;
  goff[t] = hist[t * ntiles + blockIdx.x];
  for (int k = 0; k < kSortThreads / 32; k++) wcount[k][t] = 0;
  __syncthreads();
  int base = blockIdx.x * kTile;
  unsigned lt = (1u << lane) - 1u;
  for (int r = 0; r < kTile / kSortThreads; r++) {
    int idx = base + r * kSortThreads + t;
    bool valid = idx < n;
    int key = valid ? keys_in[idx] : 0;
    int d = valid ? ((key >> shift) & 255) : 256 + lane;  // invalid lanes never match
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int wrank = __popc(peers & lt);
    if (valid && wrank == 0) wcount[w][d] = __popc(peers);
    __syncthreads();
    // per digit: exclusive prefix over warps, in warp order (stable)
    {
      int dd = t;
      int run = running[dd];
      for (int k = 0; k < kSortThreads / 32; k++) {
        int c = wcount[k][dd];
        wcount[k][dd] = run;
        run += c;
      }
      running[dd] = run;
    }
    __syncthreads();
    if (valid) {
      int pos = goff[d] + wcount[w][d] + wrank;
      keys_out[pos] = key;
      vals_out[pos] = vals_in[idx];
    }
    __syncthreads();
    for (int k = 0; k < kSortThreads / 32; k++) wcount[k][t] = 0;
    __syncthreads();
  }
}

__global__ void k_cell_ranges(const int *skeys, int n, int *cstart, int *cend) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int key = skeys[k];
  if (k == 0 || skeys[k - 1] != key) cstart[key] = k;
  if (k == n - 1 || skeys[k + 1] != key) cend[key] = k + 1;
}

// --------------------------------------------------------------- pair scan
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

// The reference's distance expression: dc = p_j - p_i; (x*x + y*y) + z*z,
// no fused multiply-add (neighbourlist.cpp:263-264, maths_vector.h:104-107).
__device__ __forceinline__ double ref_sqrdist(double xi, double yi, double zi, double xj, double yj,
                                              double zj) {
  double dx = __dsub_rn(xj, xi), dy = __dsub_rn(yj, yi), dz = __dsub_rn(zj, zi);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

template <bool FILL>
__global__ void k_nlist_scan(PackView v) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= v.n_atoms) return;
  int i = warp;
  int s = v.sys_of[i];
  const double *g = v.grid + 8 * s;
  double xi = v.x[i], yi = v.y[i], zi = v.z[i];
  double lim = v.sp[s].nl_lim2_d;
  int cx, cy, cz;
  cell_of(g, xi, yi, zi, cx, cy, cz);
  int nx = (int)g[4], ny = (int)g[5], nz = (int)g[6];
  int koff = (int)g[7];
  long long out = 0;
  if (FILL) {
    if (v.row_start[v.n_atoms] > v.nl_cap) return;  // overflow: host re-plans
    out = v.row_start[i];
  }
  int count = 0;
  unsigned lt = (1u << lane) - 1u;
  for (int dz = -1; dz <= 1; dz++) {
    int zz = cz + dz;
    if (zz < 0 || zz >= nz) continue;
    for (int dy = -1; dy <= 1; dy++) {
      int yy = cy + dy;
      if (yy < 0 || yy >= ny) continue;
      for (int dx = -1; dx <= 1; dx++) {
        int xx = cx + dx;
        if (xx < 0 || xx >= nx) continue;
        int c = koff + (zz * ny + yy) * nx + xx;
        int b = v.cell_start[c], e = v.cell_end[c];
        for (int k0 = b; k0 < e; k0 += 32) {
          int k = k0 + lane;
          bool pass = false;
          int j = 0;
          if (k < e) {
            j = v.sorted_atom[k];
            double d2 = ref_sqrdist(xi, yi, zi, v.x[j], v.y[j], v.z[j]);
            pass = !(d2 > lim) && j != i;
          }
          unsigned m = __ballot_sync(0xffffffffu, pass);
          if (FILL && pass) {
            int bo = bond_order(v, s, i, j);
            v.nl[out + count + __popc(m & lt)] = ((unsigned)j << 3) | (unsigned)bo;
          }
          count += __popc(m);
        }
      }
    }
  }
  if (!FILL && lane == 0) v.row_cnt[i] = count;
}

// --------------------------------------------------------------- scans
// exclusive scan of row_cnt (int) into row_start (int64), total at [n]
__global__ void k_scan_blocks(const int *cnt, int n, long long *out, long long *bsum) {
  __shared__ long long sh[1024];
  int t = threadIdx.x;
  int idx = blockIdx.x * 1024 + t;
  long long x = idx < n ? cnt[idx] : 0;
  sh[t] = x;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    long long val = t >= off ? sh[t - off] : 0;
    __syncthreads();
    sh[t] += val;
    __syncthreads();
  }
  if (idx < n) out[idx] = sh[t] - x;
  if (t == 1023) bsum[blockIdx.x] = sh[t];
}

__global__ void k_scan_bsum(long long *bsum, int nb, long long *total_out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    long long run = 0;
    for (int k = 0; k < nb; k++) {
      long long x = bsum[k];
      bsum[k] = run;
      run += x;
    }
    *total_out = run;
  }
}

__global__ void k_scan_add(long long *out, int n, const long long *bsum) {
  int idx = blockIdx.x * 1024 + threadIdx.x;
  if (idx < n) out[idx] += bsum[blockIdx.x];
}

__global__ void k_set_overflow(PackView v) {
  if (v.row_start[v.n_atoms] > v.nl_cap) atomicExch(&v.flags[F_NL_OVERFLOW], 1);
}

// --------------------------------------------------------------- launchers
void launch_nlist_count(Pack &p, cudaStream_t st) {
  PackView &v = p.v;
  int N = v.n_atoms;
  if (N == 0) return;
  // boxes start empty: min keys at the top of the range, max keys at 0
  cudaMemsetAsync(v.bbox, 0xFF, sizeof(unsigned long long) * 3 * v.n_sys, st);
  cudaMemsetAsync(v.bbox + 3 * v.n_sys, 0, sizeof(unsigned long long) * 3 * v.n_sys, st);
  int bb_blocks = (N + 255) / 256;
  if (bb_blocks > 592) bb_blocks = 592;
  PDGPU_LAUNCH(k_bbox, bb_blocks, 256, 0, st, v);
  PDGPU_LAUNCH(k_grid_plan, (v.n_sys + 127) / 128, 128, 0, st, v);
  int *ka = v.cell_key, *va = v.sorted_atom, *kb = p.tmp_keys, *vb = p.tmp_vals;
  PDGPU_LAUNCH(k_cell_keys, (N + 255) / 256, 256, 0, st, v, ka, va);
  int ntiles = (N + kTile - 1) / kTile;
  for (int pass = 0; pass < p.radix_passes; pass++) {
    int shift = 8 * pass;
    PDGPU_LAUNCH(k_radix_hist, ntiles, kSortThreads, 0, st, ka, N, shift, p.sort_hist, ntiles);
    PDGPU_LAUNCH(k_scan_small, 1, 1024, 0, st, p.sort_hist, 256 * ntiles);
    PDGPU_LAUNCH(k_radix_scatter, ntiles, kSortThreads, 0, st, ka, va, kb, vb, N, shift, p.sort_hist, ntiles);
    int *t1 = ka, *t2 = va;
    ka = kb;
    va = vb;
    kb = t1;
    vb = t2;
  }
  if (ka != v.cell_key) {
    cudaMemcpyAsync(v.cell_key, ka, sizeof(int) * N, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(v.sorted_atom, va, sizeof(int) * N, cudaMemcpyDeviceToDevice, st);
  }
  cudaMemsetAsync(v.cell_start, 0, sizeof(int) * v.cell_cap, st);
  cudaMemsetAsync(v.cell_end, 0, sizeof(int) * v.cell_cap, st);
  PDGPU_LAUNCH(k_cell_ranges, (N + 255) / 256, 256, 0, st, v.cell_key, N, v.cell_start, v.cell_end);
  int warps_per_block = 8;
  int blocks = (N + warps_per_block - 1) / warps_per_block;
  PDGPU_LAUNCH((k_nlist_scan<false>), blocks, 32 * warps_per_block, 0, st, v);
  int nb = (N + 1023) / 1024;
  PDGPU_LAUNCH(k_scan_blocks, nb, 1024, 0, st, v.row_cnt, N, v.row_start, p.scan_tmp);
  PDGPU_LAUNCH(k_scan_bsum, 1, 32, 0, st, p.scan_tmp, nb, v.row_start + N);
  PDGPU_LAUNCH(k_scan_add, nb, 1024, 0, st, v.row_start, N, p.scan_tmp);
  PDGPU_LAUNCH(k_set_overflow, 1, 1, 0, st, v);
}

void launch_nlist_fill(Pack &p, cudaStream_t st) {
  PackView &v = p.v;
  int N = v.n_atoms;
  if (N == 0) return;
  int warps_per_block = 8;
  int blocks = (N + warps_per_block - 1) / warps_per_block;
  PDGPU_LAUNCH((k_nlist_scan<true>), blocks, 32 * warps_per_block, 0, st, v);
  // the same pair set re-cut into cluster-pair tiles for the tile passes
  if (v.tile_mode) launch_tiles_build(v, st);
}

}  // namespace pdgpu
