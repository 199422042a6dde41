// PP kick without any device allocation by the library.
//
// Some callers cannot let a library call cudaMalloc: a driver that hands out
// every byte of device memory through its own pool, a run under an
// allocation-free execution or watchdog policy, or an embedding where the
// allocator belongs to another runtime.  cube_pp_force_noalloc serves them:
// the caller passes device-resident inputs and outputs, and all the scratch the
// PP kick needs (cell table, PP-cell counts and starts, sorted particles, work
// list, counters) lives in one file-scope device array, g_noalloc_scratch,
// sized for at most CUBE_NOALLOC_MAX_PARTICLES stored particles and
// CUBE_NOALLOC_MAX_CELLS PP cells.  Every GPU that loads this library holds the
// array until the process exits.
//
// Host code cannot use the array's name as a device address (there it is only a
// host-side stand-in), so the first call on each device looks the address up
// with cudaGetSymbolAddress while that device is current and keeps it for the
// later calls on that device; that first call belongs before any stream capture
// begins.  All calls share the one
// array and it keeps the previous call's contents: the counters are cleared on
// every call, and calls that overlap on the GPU (two streams, or two host
// threads) race on it.
#include <cstring>

#include "common.cuh"

namespace cube {

// byte budget of the shared scratch, carved in 256-byte aligned pieces
constexpr int64_t kNaParticles = CUBE_NOALLOC_MAX_PARTICLES;
constexpr int64_t kNaCells = CUBE_NOALLOC_MAX_CELLS;
constexpr int kNaTiles = 64;
constexpr int kNaSub = 4096;
constexpr int kNaSpill = 2048;

constexpr size_t na_align(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kOffCellBase = 0;                                                     // int64 [ncoarse]
constexpr size_t kOffCount = kOffCellBase + na_align(sizeof(int64_t) * kNaCells);     // int32 [cells]
constexpr size_t kOffStart = kOffCount + na_align(sizeof(int32_t) * kNaCells);         // int32 [cells + 1]
constexpr size_t kOffScan = kOffStart + na_align(sizeof(int32_t) * (kNaCells + 1));    // int32 scan scratch
constexpr size_t kOffSpos = kOffScan + na_align(sizeof(int32_t) * (kNaCells / 4096 + 2));
constexpr size_t kOffItems = kOffSpos + na_align(sizeof(float4) * kNaParticles);       // PPItem work list
constexpr size_t kItemCap = kNaCells + kNaParticles / kPPChunk + 16;
constexpr size_t kOffSpill = kOffItems + na_align(sizeof(PPItem) * kItemCap);
constexpr size_t kOffSpillRank = kOffSpill + na_align(sizeof(Spill) * kNaSpill);
constexpr size_t kOffTiles = kOffSpillRank + na_align(sizeof(int32_t) * kNaSpill);
constexpr size_t kOffRange = kOffTiles + na_align(sizeof(TilePP) * kNaTiles);
constexpr size_t kOffCounters = kOffRange + na_align(sizeof(float) * kNaSub);          // int32 [128]
constexpr size_t kNaSchedInts = 2 * 32 * kNaTiles + 2 * (kNaTiles + 1);                 // sched_ints(64)
constexpr size_t kOffSched = kOffCounters + na_align(sizeof(int32_t) * 128);            // PP schedule
constexpr size_t kNaBytes = kOffSched + na_align(sizeof(int32_t) * kNaSchedInts);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// device address of the scratch per device, looked up once per device
constexpr int kNaMaxDevices = 64;
static unsigned char *g_na_addr[kNaMaxDevices] = {};

size_t noalloc_scratch_bytes() { return kNaBytes; }

// The per-call tables (PP grid per tile, PP range per subtile) travel to the scratch as a
// kernel argument, so no copy on the GPU reads this call's host stack after it returns.
struct NaTables {
  TilePP tiles[kNaTiles];
  float range[kNaSub];
  int32_t ntile, nsub;
};
static_assert(sizeof(NaTables) <= 32000, "kernel parameter space (32764 bytes on sm_70 and later)");

__global__ void k_na_tables(const NaTables t, TilePP *tiles, float *range) {
  for (int i = threadIdx.x; i < t.ntile; i += blockDim.x) tiles[i] = t.tiles[i];
  for (int i = threadIdx.x; i < t.nsub; i += blockDim.x) range[i] = t.range[i];
}

int pp_force_noalloc(const Lay &L, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                     const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp,
                     int64_t n_used, float *d_vp, float mass, float a_mid, float dt, float *d_out,
                     cudaStream_t s) {
  if (!ires || !ixyz3 || !apm3 || !ratio_sf || !d_rhoc || !d_idx_b_r || !d_xp || !d_vp || !d_out)
    return CUBE_ERR_INVALID;
  if (n_used < 0 || n_used > kNaParticles) return CUBE_ERR_CAPACITY;
  if (L.ntile > kNaTiles || L.ns3 > kNaSub) return CUBE_ERR_CAPACITY;
  if ((int64_t)L.ntile * L.nte * L.nte * L.nte > kNaCells) return CUBE_ERR_CAPACITY;
  for (int l = 0; l < 7; l++)
    if (ratio_sf[l] < 1 || ratio_sf[l] > 64) return CUBE_ERR_INVALID;

  // per-subtile tables by location (pp_force_kernel.cu:987-1004), on the stack
  int ires_loc[kNaSub];
  bool seen[kNaSub];
  NaTables tab;
  float *range_loc = tab.range;
  TilePP *tiles = tab.tiles;
  tab.ntile = L.ntile;
  tab.nsub = L.ns3;
  for (int q = 0; q < L.ns3; q++) seen[q] = false;
  for (int it = 0; it < L.ns3; it++) {
    const int *r = ixyz3 + 6 * it;
    const int sx = r[0] - 1, sy = r[1] - 1, sz = r[2] - 1, tx = r[3] - 1, ty = r[4] - 1, tz = r[5] - 1;
    if (sx < 0 || sx >= L.nns || sy < 0 || sy >= L.nns || sz < 0 || sz >= L.nns || tx < 0 || tx >= L.nnt ||
        ty < 0 || ty >= L.nnt || tz < 0 || tz >= L.nnt || ires[it] < 2 || ires[it] > 6)
      return CUBE_ERR_INVALID;
    const int loc = (((tz * L.nnt + ty) * L.nnt + tx) * L.nns + sz) * L.nns * L.nns + sy * L.nns + sx;
    if (seen[loc]) return CUBE_ERR_INVALID;
    seen[loc] = true;
    ires_loc[loc] = ires[it];
    range_loc[loc] = apm3[ires[it] - 1];
  }
  int64_t ncells = 0, interior = 0;
  int max_rcp = 1;
  const int nss = L.nns * L.nns * L.nns;
  for (int t = 0; t < L.ntile; t++) {
    int rcp = ratio_sf[1];
    for (int q = 0; q < nss; q++) rcp = rcp > ratio_sf[ires_loc[t * nss + q] - 1] ? rcp : ratio_sf[ires_loc[t * nss + q] - 1];
    tiles[t].rcp = rcp;
    tiles[t].S = rcp * (L.nt + 2);
    tiles[t].cell0 = ncells;
    ncells += (int64_t)tiles[t].S * tiles[t].S * tiles[t].S;
    interior += (int64_t)L.nt * rcp * L.nt * rcp * L.nt * rcp;
    max_rcp = rcp > max_rcp ? rcp : max_rcp;
  }
  if (ncells > kNaCells) return CUBE_ERR_CAPACITY;
  if (interior + n_used / kPPChunk + 16 > (int64_t)kItemCap) return CUBE_ERR_CAPACITY;
  if (bin_smem_bytes(max_rcp) > 200 * 1024) return CUBE_ERR_INVALID;
  if (sched_ints(L.ntile) > kNaSchedInts) return CUBE_ERR_CAPACITY;

  // device address of the scratch on the current device (once per device)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) return CUBE_ERR_CUDA;
  if (!g_na_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CUBE_ERR_CUDA;
    g_na_addr[dev] = (unsigned char *)p;
  }
  unsigned char *base = g_na_addr[dev];
  int64_t *cell_base = (int64_t *)(base + kOffCellBase);
  int32_t *count = (int32_t *)(base + kOffCount);
  int32_t *cell_start = (int32_t *)(base + kOffStart);
  int32_t *scan_tmp = (int32_t *)(base + kOffScan);
  float4 *spos = (float4 *)(base + kOffSpos);
  PPItem *items = (PPItem *)(base + kOffItems);
  Spill *spill = (Spill *)(base + kOffSpill);
  int32_t *spill_rank = (int32_t *)(base + kOffSpillRank);
  TilePP *d_tiles = (TilePP *)(base + kOffTiles);
  float *d_range = (float *)(base + kOffRange);
  int32_t *ctr = (int32_t *)(base + kOffCounters);  // [0] spill_n [2] err
  int32_t *sched = (int32_t *)(base + kOffSched);    // zeroed by launch_pp_items

  // the scratch keeps the previous call's contents: reset what must start at zero
  if (cudaMemsetAsync(ctr, 0, sizeof(int32_t) * 128, s) != cudaSuccess) return CUBE_ERR_CUDA;
  if (cudaMemsetAsync(d_out, 0, sizeof(float) * 6, s) != cudaSuccess) return CUBE_ERR_CUDA;
  k_na_tables<<<1, 256, 0, s>>>(tab, d_tiles, d_range);

  launch_cell_table(L, d_rhoc, d_idx_b_r, cell_base, s);
  BinArgs b{};
  b.L = &L;
  b.d_tiles = d_tiles;
  b.max_rcp = max_rcp;
  b.ncells = ncells;
  b.xp = d_xp;
  b.rhoc = d_rhoc;
  b.cell_base = cell_base;
  b.count = count;
  b.cell_start = cell_start;
  b.spos = spos;
  b.spill = spill;
  b.spill_rank = spill_rank;
  b.spill_n = ctr;
  b.spill_cap = kNaSpill;
  b.scan_tmp = scan_tmp;
  b.err = ctr + 2;
  b.spatial = 1;
  launch_pp_binning(b, s);
  int num_sms = 148;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  PPArgs p{};
  p.L = &L;
  p.d_tiles = d_tiles;
  p.h_tiles = tiles;
  p.ncells = ncells;
  p.cell_start = cell_start;
  p.spos = spos;
  p.range_loc = d_range;
  p.items = items;
  p.sched = sched;
  p.item_cap = (int64_t)kItemCap;
  p.vp = d_vp;
  p.mass2 = mass * mass;
  p.kick = (float)((double)(a_mid * dt / 6.0f) / 3.14159265358979323846);
  p.out = d_out;
  p.want_vmax = 1;
  p.err = ctr + 2;
  p.num_sms = num_sms;
  p.pairs = nullptr;
  launch_pp_items(p, s);
  launch_pp_force(p, s);
  // device-side failure mask next to the outputs (word 5)
  if (cudaMemcpyAsync(d_out + 5, ctr + 2, sizeof(int32_t), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return CUBE_ERR_CUDA;
  if (cudaGetLastError() != cudaSuccess) return CUBE_ERR_CUDA;
  return CUBE_OK;
}

}  // namespace cube
