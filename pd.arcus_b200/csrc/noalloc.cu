// Neighbour-list build that allocates no device memory.
//
// For callers that cannot allocate: host frameworks that own all device
// memory themselves (a fixed pool reserved at start-up) and forbid
// allocation after it.  The caller passes inputs and outputs; every scratch
// buffer of the build lives in one file-scope static __device__ array, sized
// for at most kNoAllocMaxAtoms atoms.
//
// The array is part of the library image: every GPU that loads libpdgpu
// holds it until the process exits.  All calls share it and it keeps the
// last call's contents, so calls that overlap on the GPU (two streams, or
// two host threads) race and must be serialised by the caller.  Whatever
// must start at zero is cleared by each call.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>

#include "internal.cuh"

namespace pdgpu {

constexpr int kNoAllocMaxAtoms = 65536;
namespace {
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr int kCellCap = 2 * kNoAllocMaxAtoms + 64;
constexpr int kTiles = (kNoAllocMaxAtoms + 2047) / 2048;
constexpr int kScanLen = (kNoAllocMaxAtoms + 1023) / 1024 + 2;
// byte offsets of the regions inside the scratch array
constexpr size_t kOffSysOf = 0;
constexpr size_t kOffOffPtr = kOffSysOf + align256(sizeof(int) * kNoAllocMaxAtoms);
constexpr size_t kOffRowCnt = kOffOffPtr + align256(sizeof(int) * (kNoAllocMaxAtoms + 1));
constexpr size_t kOffKeys = kOffRowCnt + align256(sizeof(int) * kNoAllocMaxAtoms);
constexpr size_t kOffVals = kOffKeys + align256(sizeof(int) * kNoAllocMaxAtoms);
constexpr size_t kOffTmpKeys = kOffVals + align256(sizeof(int) * kNoAllocMaxAtoms);
constexpr size_t kOffTmpVals = kOffTmpKeys + align256(sizeof(int) * kNoAllocMaxAtoms);
constexpr size_t kOffCellStart = kOffTmpVals + align256(sizeof(int) * kNoAllocMaxAtoms);
constexpr size_t kOffCellEnd = kOffCellStart + align256(sizeof(int) * kCellCap);
constexpr size_t kOffHist = kOffCellEnd + align256(sizeof(int) * kCellCap);
constexpr size_t kOffScan = kOffHist + align256(sizeof(int) * 256 * kTiles);
constexpr size_t kOffGrid = kOffScan + align256(sizeof(long long) * kScanLen);
constexpr size_t kOffBbox = kOffGrid + align256(sizeof(double) * 8);
constexpr size_t kOffFlags = kOffBbox + align256(sizeof(unsigned long long) * 6);
constexpr size_t kOffSmall = kOffFlags + align256(sizeof(int) * F_COUNT);  // atom_off[2], mid, band_off
constexpr size_t kOffParams = kOffSmall + 256;
constexpr size_t kScratchBytes = kOffParams + align256(sizeof(SysParams));
}  // namespace

// About 2.9 MB.
static __device__ __align__(256) unsigned char g_nlist_scratch[kScratchBytes];

// Device addresses of the array, looked up once per device (host code may
// not use the symbol itself: on the host it names a stand-in object).  The
// lookup runs under a lock; the filled entries are read without it.
static std::atomic<void *> g_scratch_dev[64];
static std::mutex g_scratch_lock;

static int scratch_address(int device, unsigned char **out) {
  if (device < 0 || device >= 64) {
    set_error("device index out of range");
    return PDGPU_ERR_ARG;
  }
  void *p = g_scratch_dev[device].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_scratch_lock);
    p = g_scratch_dev[device].load(std::memory_order_relaxed);
    if (!p) {
      // with lazy module loading (CUDA_MODULE_LOADING=LAZY, the default)
      // this first lookup on a device loads the module that holds the
      // array, which is when the device memory for it is taken
      cudaError_t e = cudaGetSymbolAddress(&p, g_nlist_scratch);
      if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(nlist scratch)");
      g_scratch_dev[device].store(p, std::memory_order_release);
    }
  }
  *out = (unsigned char *)p;
  return PDGPU_OK;
}

// Load the array's module on the current device and look its address up
// (pdgpu_ctx_create calls this, so a caller that creates its context before
// reserving its memory pool has the array in place before the pool).
int noalloc_prepare_current_device() {
  int device = 0;
  cudaError_t ce = cudaGetDevice(&device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaGetDevice");
  unsigned char *base = nullptr;
  return scratch_address(device, &base);
}

// (j << 3 | bondorder) -> the reference's packed entry j | bondorder << 24
__global__ void k_entries_to_reference(unsigned *e, long long n) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k < n) {
    unsigned x = e[k];
    e[k] = ((x >> 3) & 0x00FFFFFFu) | ((x & 7u) << 24);
  }
}

}  // namespace pdgpu

using namespace pdgpu;

extern "C" int pdgpu_nlist_build_noalloc(const double *x, const double *y, const double *z, int32_t natoms,
                                         double list_cutoff, int32_t max_index_delta, const int8_t *band,
                                         const int32_t *offdiag_ptr, const int32_t *offdiag_pairs,
                                         int64_t *row_start, uint32_t *entries, int64_t capacity,
                                         int64_t *count, void *stream) {
  if (natoms <= 0 || natoms > kNoAllocMaxAtoms) {
    set_error("pdgpu_nlist_build_noalloc: natoms must be in [1, " + std::to_string(kNoAllocMaxAtoms) +
              "] (the size of its static scratch); use pdgpu_nlist_build for larger systems");
    return PDGPU_ERR_ARG;
  }
  if (!x || !y || !z || !row_start || !count || (natoms > 1 && !band) || max_index_delta < 1 ||
      !(list_cutoff > 0) || capacity < 0 || (capacity > 0 && !entries) || (!offdiag_ptr != !offdiag_pairs)) {
    set_error("pdgpu_nlist_build_noalloc: bad arguments");
    return PDGPU_ERR_ARG;
  }
  int device = 0;
  cudaError_t ce = cudaGetDevice(&device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaGetDevice");
  unsigned char *base = nullptr;
  int r = scratch_address(device, &base);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;

  // a Pack whose buffers are the static scratch and the caller's arrays;
  // it owns nothing (no allocations to free)
  Pack p;
  p.device = device;
  PackView &v = p.v;
  v.n_atoms = natoms;
  v.n_sys = 1;
  int *small = (int *)(base + kOffSmall);
  v.atom_off = small;                            // [2]
  v.mid = small + 2;                             // [1]
  v.band_off = (const long long *)(small + 4);   // [1], 8-byte aligned
  v.sys_of = (const int *)(base + kOffSysOf);
  v.sp = (const SysParams *)(base + kOffParams);
  v.x = (double *)x;
  v.y = (double *)y;
  v.z = (double *)z;
  v.band = band;
  v.off_ptr = offdiag_ptr ? offdiag_ptr : (const int *)(base + kOffOffPtr);
  v.off_data = offdiag_pairs ? (const int2 *)offdiag_pairs : nullptr;
  v.row_start = (long long *)row_start;
  v.row_cnt = (int *)(base + kOffRowCnt);
  v.nl = (unsigned *)entries;
  v.nl_cap = capacity;
  v.cell_key = (int *)(base + kOffKeys);
  v.sorted_atom = (int *)(base + kOffVals);
  v.cell_start = (int *)(base + kOffCellStart);
  v.cell_end = (int *)(base + kOffCellEnd);
  v.cell_cap = 2 * natoms + 64;
  v.grid = (double *)(base + kOffGrid);
  v.bbox = (unsigned long long *)(base + kOffBbox);
  v.flags = (int *)(base + kOffFlags);
  p.tmp_keys = (int *)(base + kOffTmpKeys);
  p.tmp_vals = (int *)(base + kOffTmpVals);
  p.sort_hist = (int *)(base + kOffHist);
  p.scan_tmp = (long long *)(base + kOffScan);
  int bits = 1;
  while ((1LL << bits) < (long long)v.cell_cap) bits++;
  p.radix_passes = (bits + 7) / 8;

  // per-call state: what must start at zero is cleared here
  SysParams sp;
  memset(&sp, 0, sizeof sp);
  sp.nl_lim2_d = list_cutoff * list_cutoff;
  struct {
    int atom_off[2];
    int mid;
    int pad;
    long long band_off;
  } hs = {{0, natoms}, max_index_delta, 0, 0};
  PDGPU_CUDA(cudaMemcpyAsync(small, &hs, sizeof hs, cudaMemcpyHostToDevice, st));
  PDGPU_CUDA(cudaMemcpyAsync((void *)v.sp, &sp, sizeof sp, cudaMemcpyHostToDevice, st));
  PDGPU_CUDA(cudaMemsetAsync((void *)v.sys_of, 0, sizeof(int) * natoms, st));
  PDGPU_CUDA(cudaMemsetAsync(v.flags, 0, sizeof(int) * F_COUNT, st));
  if (!offdiag_ptr) PDGPU_CUDA(cudaMemsetAsync((void *)v.off_ptr, 0, sizeof(int) * (natoms + 1), st));

  launch_nlist_count(p, st);
  long long total = 0;
  PDGPU_CUDA(cudaMemcpyAsync(&total, row_start + natoms, sizeof total, cudaMemcpyDeviceToHost, st));
  PDGPU_CUDA(cudaStreamSynchronize(st));
  *count = total;
  if (total > capacity) {
    set_error("pdgpu_nlist_build_noalloc: entries capacity " + std::to_string(capacity) + " < " +
              std::to_string(total) + " entries needed");
    return PDGPU_ERR_ARG;
  }
  launch_nlist_fill(p, st);
  if (total > 0)
    PDGPU_LAUNCH(k_entries_to_reference, (unsigned)((total + 255) / 256), 256, 0, st, (unsigned *)entries, total);
  ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return cuda_fail(ce, "pdgpu_nlist_build_noalloc");
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return cuda_fail(ce, "pdgpu_nlist_build_noalloc");
  return PDGPU_OK;
}
