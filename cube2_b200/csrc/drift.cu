// Drift of one periodic image and the rebuild of its buffers on the device:
// drift.f90:1-161 (fixed-point drift, re-binning by coarse cell, compaction) followed by
// buffer_grid.f90:13-155 and buffer_particle.f90:23-345 (periodic buffer cells, which
// hold copies of the particles of the physical cells they mirror).
//
// The reference visits each tile's stored copies (physical and buffer) layer by layer
// (source row k modulo nlayer), then in storage order, and appends every copy that lands
// in the tile's physical region to its destination cell (drift.f90:94-118).  The order
// inside a destination cell is thus by (ilayer of the source row, storage index), and
// every destination's particles come from a few nearby source cells of one tile.  Here:
//
//   k_drift_runs   warp per source cell: the destination of each copy; the copies of the
//                  cell that share a destination form a run (at most 64 per source cell),
//                  and each copy gets its rank inside its run (warp ballots, in storage
//                  order); runs go to a flat table with the reference's visiting key.
//   k_ext_counts   new counts of every extended cell (buffer cells mirror physical ones),
//   k_row_sums,
//   k_scan_rows    and the new spine idx_b_r (one inclusive scan over the rows).
//   k_runs_fill    runs grouped by destination cell (counting sort on the destination),
//   k_runs_order   and each run's first slot: the destination cell's start plus the
//                  particles of the runs with a smaller key (runs per cell are few).
//   k_drift_write  warp per source cell again: every kept copy writes its new offset
//                  (xp + nint(dt vp / (x_res ratio_cs)), int16 wrap), vp and pid to its slot.
//   k_halo_fill    warp per buffer cell: copy of the mirrored physical cell.
//
// Everything is linear in the particles and deterministic (no order depends on atomics).
#include "common.cuh"

namespace cube {

struct DriftRun {
  int32_t dest;   // physical coarse cell of the image, (z * nc + y) * nc + x
  int32_t count;  // copies of the source cell that land there
  uint64_t key;   // ilayer(source row) << 32 | source cell: the reference's visiting order
};

constexpr int kDriftMaxRuns = 64;    // destination cells of one source cell
constexpr int kRankBits = 26;        // run slot word: entry << 26 | rank inside the run
constexpr uint32_t kDropped = 0xffffffffu;
constexpr int kDriftWarps = 8;
// Run-table slots are reserved per warp kRunChunk at a time (one atomic per chunk instead of
// one per source cell on a single counter); the unused end of a chunk holds dest = -1.
constexpr int kRunChunk = 64;
static_assert(kRunChunk >= kDriftMaxRuns, "a cell's runs fit one chunk");
constexpr int kDriftGridPerSM = 16;  // blocks per SM of the warp-per-cell kernels (at most)

struct DriftK {
  int nt, ncb, nte, nnt, nc, nlayer, tile_periodic;
  int64_t ncells_src;  // ntile * nte^3 extended cells
  int64_t n_used, n_used_new;  // stored copies of the current / new image (bounds of the spines)
  float dt_mid, rcs_f;
  double xres_rcs;     // x_resolution * ratio_cs
  const int32_t *rhoc;
  const int64_t *cell_base;
  const int16_t *xp;
  const float *vp;
  const int64_t *pid;
  uint32_t *runrank;     // [n_used] run slot word of each stored copy
  int32_t *run_base;     // [ncells_src] first run of each source cell
  DriftRun *runs;
  int32_t run_cap;
  int32_t *ctr;          // [0] runs, [1] kept copies
  int32_t *dest_runs;    // [nc^3] runs per destination
  int32_t *phys_count;   // [nc^3] particles per destination
  int32_t *err;
  // second half
  const int32_t *dest_start;  // [nc^3 + 1]
  int32_t *cursor;            // [nc^3]
  int32_t *run_list;          // [runs] grouped by destination
  int64_t *run_off;           // [runs] first slot of each run
  const int64_t *cell_base_new;
  int16_t *xp_new;
  float *vp_new;
  int64_t *pid_new;
};

__device__ __forceinline__ void cell_of(const DriftK &p, int64_t S, int &t, int &cx, int &cy, int &cz) {
  const int64_t n3 = (int64_t)p.nte * p.nte * p.nte;
  t = (int)(S / n3);
  int64_t r = S - (int64_t)t * n3;
  cz = (int)(r / (p.nte * p.nte));
  r -= (int64_t)cz * p.nte * p.nte;
  cy = (int)(r / p.nte);
  cx = (int)(r - (int64_t)cy * p.nte);
}

// drift.f90:57-66: destination of a stored copy, or -1 when it leaves the tile's physical
// region.  xq = (i-1) + (u+0.5) 2^-16 is exact in double; deltax = (dt_mid*vp)/ratio_cs
// in float; ig = ceiling(xq + deltax) in [1, nt] <=> 0 < xq + deltax <= nt.
__device__ __forceinline__ int32_t drift_dest(const DriftK &p, int64_t ip, int cx, int cy, int cz, int t) {
  const int c[3] = {cx, cy, cz};
  const int tt[3] = {t % p.nnt, (t / p.nnt) % p.nnt, t / (p.nnt * p.nnt)};
  int g[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double frac = ((double)(uint16_t)p.xp[3 * ip + d] + 0.5) * (1.0 / 65536.0);
    const double xq = (double)(c[d] - p.ncb) + frac;
    const float dl = __fdiv_rn(__fmul_rn(p.dt_mid, p.vp[3 * ip + d]), p.rcs_f);
    const double s = __dadd_rn(xq, (double)dl);
    if (!(s > 0.0 && s <= (double)p.nt)) return -1;
    g[d] = tt[d] * p.nt + (int)ceil(s) - 1;
  }
  return (g[2] * p.nc + g[1]) * p.nc + g[0];
}

__global__ void __launch_bounds__(kDriftWarps * 32) k_drift_runs(DriftK p) {
  __shared__ int32_t s_dest[kDriftWarps][kDriftMaxRuns];
  __shared__ int32_t s_cnt[kDriftWarps][kDriftMaxRuns];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int32_t *td = s_dest[warp], *tc = s_cnt[warp];
  const unsigned lt = (1u << lane) - 1u;
  const int64_t stride = (int64_t)gridDim.x * kDriftWarps;
  int64_t S = (int64_t)blockIdx.x * kDriftWarps + warp;
  // the count and first slot of the next cell are loaded one cell ahead
  int n_next = S < p.ncells_src ? p.rhoc[S] : 0;
  int64_t base_next = S < p.ncells_src ? p.cell_base[S] : 0;
  int cur = 0, end = 0;  // this warp's reserved run slots [cur, end)
  int kept_w = 0;        // kept copies counted by this lane
  auto close_chunk = [&]() {
    for (int e = cur + lane; e < end; e += 32)
      if (e < p.run_cap) p.runs[e].dest = -1;
  };
  for (; S < p.ncells_src; S += stride) {
    const int n = n_next;
    const int64_t base = base_next;
    if (S + stride < p.ncells_src) {
      n_next = p.rhoc[S + stride];
      base_next = p.cell_base[S + stride];
    }
    if (n <= 0) continue;
    if (n >= (1 << kRankBits) - 1) {  // the rank field holds ranks below 2^26 - 1
      if (lane == 0) atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
      continue;
    }
    if (base < 0 || base + n > p.n_used) {  // the spine does not match the counts
      if (lane == 0) atomicOr(p.err, 1 << CUBE_ERR_INVALID);
      continue;
    }
    int t, cx, cy, cz;
    cell_of(p, S, t, cx, cy, cz);
    int nent = 0;  // warp-uniform
    // 64 copies per step: the loads of both halves are in flight together
    for (int c64 = 0; c64 < n; c64 += 64) {
    const int32_t D2[2] = {c64 + lane < n ? drift_dest(p, base + c64 + lane, cx, cy, cz, t) : -1,
                           c64 + 32 + lane < n ? drift_dest(p, base + c64 + 32 + lane, cx, cy, cz, t) : -1};
    for (int h = 0; h < 2 && c64 + 32 * h < n; h++) {
      const int c0 = c64 + 32 * h;
      const int l = c0 + lane;
      const int32_t D = D2[h];
      uint32_t word = kDropped;
      unsigned pending = __ballot_sync(0xffffffffu, D >= 0);
      while (pending) {
        const int32_t Dl = __shfl_sync(0xffffffffu, D, __ffs(pending) - 1);
        const unsigned grp = __ballot_sync(0xffffffffu, D == Dl);
        const unsigned h0 = __ballot_sync(0xffffffffu, lane < nent && td[lane] == Dl);
        const unsigned h1 = __ballot_sync(0xffffffffu, lane + 32 < nent && td[lane + 32] == Dl);
        int e = h0 ? __ffs(h0) - 1 : (h1 ? 31 + __ffs(h1) : -1);
        if (e < 0 && nent < kDriftMaxRuns) {
          e = nent++;
          if (lane == 0) {
            td[e] = Dl;
            tc[e] = 0;
          }
          __syncwarp();
        }
        if (e >= 0) {
          const int prior = tc[e];
          if ((grp >> lane) & 1u) word = ((uint32_t)e << kRankBits) | (uint32_t)(prior + __popc(grp & lt));
          __syncwarp();
          if (lane == 0) tc[e] = prior + __popc(grp);
          __syncwarp();
        } else if (lane == 0) {
          atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);  // more than kDriftMaxRuns destinations
        }
        pending &= ~grp;
      }
      if (l < n) p.runrank[base + l] = word;
    }
    }
    if (nent) {
      if (cur + nent > end) {  // a new chunk of run slots
        close_chunk();
        int c = 0;
        if (lane == 0) c = atomicAdd(&p.ctr[0], kRunChunk);
        cur = __shfl_sync(0xffffffffu, c, 0);
        end = cur + kRunChunk;
      }
      const int rb = cur;
      cur += nent;
      if (lane == 0) p.run_base[S] = rb;
      const uint64_t key = ((uint64_t)(cz % p.nlayer) << 32) | (uint64_t)S;
      int kept = 0;
      for (int e = lane; e < nent; e += 32) {
        if (rb + e < p.run_cap) {
          DriftRun r;
          r.dest = td[e];
          r.count = tc[e];
          r.key = key;
          p.runs[rb + e] = r;
          atomicAdd(&p.dest_runs[r.dest], 1);
          atomicAdd(&p.phys_count[r.dest], r.count);
          kept += r.count;
        } else {
          atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
        }
      }
      kept_w += kept;
      __syncwarp();  // the table is reused by the next cell
    }
  }
  close_chunk();
  kept_w = __reduce_add_sync(0xffffffffu, kept_w);
  if (lane == 0 && kept_w) atomicAdd(&p.ctr[1], kept_w);
}

// physical cell mirrored by extended cell (t, cx, cy, cz): the image's periodic neighbour
// (buffer_grid.f90:22-40), or the tile's own periodic image for independent periodic tiles
__device__ __forceinline__ int32_t mirrored_cell(const DriftK &p, int t, int cx, int cy, int cz) {
  const int c[3] = {cx, cy, cz};
  const int tt[3] = {t % p.nnt, (t / p.nnt) % p.nnt, t / (p.nnt * p.nnt)};
  int g[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    int l = c[d] - p.ncb;
    if (p.tile_periodic) {
      l = ((l % p.nt) + p.nt) % p.nt;
      g[d] = tt[d] * p.nt + l;
    } else {
      const int x = tt[d] * p.nt + l;
      g[d] = ((x % p.nc) + p.nc) % p.nc;
    }
  }
  return (g[2] * p.nc + g[1]) * p.nc + g[0];
}

// extended cell index of a physical cell in the tile that owns it
__device__ __forceinline__ int64_t owner_ext_cell(const DriftK &p, int32_t G) {
  const int gx = G % p.nc, gy = (G / p.nc) % p.nc, gz = G / (p.nc * p.nc);
  const int t = ((gz / p.nt) * p.nnt + gy / p.nt) * p.nnt + gx / p.nt;
  const int lx = gx % p.nt + p.ncb, ly = gy % p.nt + p.ncb, lz = gz % p.nt + p.ncb;
  return (int64_t)t * p.nte * p.nte * p.nte + ((int64_t)lz * p.nte + ly) * p.nte + lx;
}

__global__ void k_ext_counts(DriftK p, const int32_t *phys_count, int32_t *rhoc_new) {
  const int64_t E = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (E >= p.ncells_src) return;
  int t, cx, cy, cz;
  cell_of(p, E, t, cx, cy, cz);
  rhoc_new[E] = phys_count[mirrored_cell(p, t, cx, cy, cz)];
}

__global__ void k_row_sums(const int32_t *rhoc, int64_t nrows, int nte, int64_t *rows) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  int64_t s = 0;
  for (int i = 0; i < nte; i++) s += rhoc[r * nte + i];
  rows[r] = s;
}

// inclusive scan of the row sums (one block): the spine idx_b_r (variables.f90:184-195)
__global__ void __launch_bounds__(1024) k_scan_rows(const int64_t *rows, int64_t nrows, int64_t *idx_b_r,
                                                    int64_t *total) {
  __shared__ int64_t ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t carry = 0;
  for (int64_t r0 = 0; r0 < nrows; r0 += 1024) {
    const int64_t r = r0 + threadIdx.x;
    int64_t x = r < nrows ? rows[r] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int64_t w = ws[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      ws[lane] = w;
    }
    __syncthreads();
    const int64_t incl = x + (warp ? ws[warp - 1] : 0) + carry;
    if (r < nrows) idx_b_r[r] = incl;
    carry += ws[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_runs_fill(DriftK p, int32_t nruns) {
  const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nruns) return;
  const int32_t D = p.runs[r].dest;
  if (D < 0) return;  // an unused slot at the end of a warp's chunk
  const int32_t slot = atomicAdd(&p.cursor[D], 1);
  p.run_list[p.dest_start[D] + slot] = r;
}

// warp per destination cell: first slot of each of its runs = the cell's start plus the
// particles of its runs with a smaller visiting key
__global__ void __launch_bounds__(kDriftWarps * 32) k_runs_order(DriftK p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ndest = (int64_t)p.nc * p.nc * p.nc;
  for (int64_t D = (int64_t)blockIdx.x * kDriftWarps + warp; D < ndest; D += (int64_t)gridDim.x * kDriftWarps) {
    const int s0 = p.dest_start[D], m = p.dest_start[D + 1] - s0;
    if (m == 0) continue;
    const int64_t start = p.cell_base_new[owner_ext_cell(p, (int32_t)D)];
    for (int i = lane; i < m; i += 32) {
      const int32_t r = p.run_list[s0 + i];
      const uint64_t key = p.runs[r].key;
      int64_t off = 0;
      for (int j = 0; j < m; j++) {
        const DriftRun o = p.runs[p.run_list[s0 + j]];
        off += o.key < key ? o.count : 0;
      }
      p.run_off[r] = start + off;
    }
  }
}

// drift.f90:111: xp + nint(dt_mid*vp / (x_resolution*ratio_cs)), stored in int16 (wraps)
__device__ __forceinline__ int16_t drift_offset(const DriftK &p, int16_t x, float v, int32_t *err) {
  const double q = __ddiv_rn((double)__fmul_rn(p.dt_mid, v), p.xres_rcs);
  if (!(fabs(q) < 2147483647.0)) {  // nint beyond the default integer: undefined in the reference
    atomicOr(err, 1 << CUBE_ERR_INVALID);
    return x;
  }
  const long long n = llround(q);
  return (int16_t)(uint16_t)((uint32_t)(int32_t)x + (uint32_t)n);
}

__global__ void __launch_bounds__(kDriftWarps * 32) k_drift_write(DriftK p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * kDriftWarps;
  int64_t S = (int64_t)blockIdx.x * kDriftWarps + warp;
  int n_next = S < p.ncells_src ? p.rhoc[S] : 0;
  int64_t base_next = S < p.ncells_src ? p.cell_base[S] : 0;
  for (; S < p.ncells_src; S += stride) {
    const int n = n_next;
    const int64_t base = base_next;
    if (S + stride < p.ncells_src) {
      n_next = p.rhoc[S + stride];
      base_next = p.cell_base[S + stride];
    }
    if (n <= 0 || n >= (1 << kRankBits) - 1) continue;
    if (base < 0 || base + n > p.n_used) continue;
    const int rb = p.run_base[S];
    for (int l = lane; l < n; l += 32) {
      const int64_t ip = base + l;
      const uint32_t w = p.runrank[ip];
      // the copy's own data does not depend on its slot: loaded beside the slot lookup
      float v[3];
      int16_t x[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        v[d] = p.vp[3 * ip + d];
        x[d] = p.xp[3 * ip + d];
      }
      const int64_t id = p.pid ? p.pid[ip] : 0;
      if (w == kDropped) continue;
      const int64_t pos = p.run_off[rb + (int)(w >> kRankBits)] + (int64_t)(w & ((1u << kRankBits) - 1u));
#pragma unroll
      for (int d = 0; d < 3; d++) {
        p.xp_new[3 * pos + d] = drift_offset(p, x[d], v[d], p.err);
        p.vp_new[3 * pos + d] = v[d];
      }
      if (p.pid) p.pid_new[pos] = id;
    }
  }
}

// warp per buffer cell: the particles of the physical cell it mirrors, in order
// (buffer_particle.f90:44-345); xp/pid may be null (velocity-only refresh, buffer_v)
__global__ void __launch_bounds__(kDriftWarps * 32) k_halo_fill(DriftK p, const int32_t *rhoc,
                                                                  const int64_t *cell_base, int16_t *xp, float *vp,
                                                                  int64_t *pid) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int64_t E = (int64_t)blockIdx.x * kDriftWarps + warp; E < p.ncells_src; E += (int64_t)gridDim.x * kDriftWarps) {
    int t, cx, cy, cz;
    cell_of(p, E, t, cx, cy, cz);
    const int lo = p.ncb, hi = p.ncb + p.nt;
    if (cx >= lo && cx < hi && cy >= lo && cy < hi && cz >= lo && cz < hi) continue;  // physical
    const int n = rhoc[E];
    if (n <= 0) continue;
    const int64_t dst = cell_base[E];
    const int64_t src = cell_base[owner_ext_cell(p, mirrored_cell(p, t, cx, cy, cz))];
    if (dst < 0 || src < 0 || dst + n > p.n_used_new || src + n > p.n_used_new) continue;  // inconsistent spine
    for (int l = lane; l < n; l += 32) {
      if (xp) {
        xp[3 * (dst + l) + 0] = xp[3 * (src + l) + 0];
        xp[3 * (dst + l) + 1] = xp[3 * (src + l) + 1];
        xp[3 * (dst + l) + 2] = xp[3 * (src + l) + 2];
      }
      vp[3 * (dst + l) + 0] = vp[3 * (src + l) + 0];
      vp[3 * (dst + l) + 1] = vp[3 * (src + l) + 1];
      vp[3 * (dst + l) + 2] = vp[3 * (src + l) + 2];
      if (pid) pid[dst + l] = pid[src + l];
    }
  }
}

static DriftK make_driftk(const DriftArgs &a) {
  const Lay &L = *a.L;
  DriftK p{};
  p.nt = L.nt;
  p.ncb = L.ncb;
  p.nte = L.nte;
  p.nnt = L.nnt;
  p.nc = L.nc;
  p.nlayer = a.nlayer;
  p.tile_periodic = L.pm3_mode == CUBE_PM3_TILE_PERIODIC;
  p.ncells_src = (int64_t)L.ntile * L.nte * L.nte * L.nte;
  p.n_used = a.n_used;
  p.n_used_new = a.n_used_new;
  p.dt_mid = a.dt_mid;
  p.rcs_f = (float)L.rcs;
  p.xres_rcs = (1.0 / 65536.0) * (double)L.rcs;
  p.rhoc = a.rhoc;
  p.cell_base = a.cell_base;
  p.xp = a.xp;
  p.vp = a.vp;
  p.pid = a.pid;
  p.runrank = a.runrank;
  p.run_base = a.run_base;
  p.runs = (DriftRun *)a.runs;
  p.run_cap = a.run_cap;
  p.ctr = a.ctr;
  p.dest_runs = a.dest_runs;
  p.phys_count = a.phys_count;
  p.err = a.err;
  p.dest_start = a.dest_start;
  p.cursor = a.cursor;
  p.run_list = a.run_list;
  p.run_off = a.run_off;
  p.cell_base_new = a.cell_base_new;
  p.xp_new = a.xp_new;
  p.vp_new = a.vp_new;
  p.pid_new = a.pid_new;
  return p;
}

size_t drift_run_bytes() { return sizeof(DriftRun); }
int64_t drift_run_slack(int num_sms) { return (int64_t)num_sms * kDriftGridPerSM * kDriftWarps * kRunChunk; }

static unsigned warp_grid(int64_t items, int num_sms) {
  const int64_t blocks = (items + kDriftWarps - 1) / kDriftWarps;
  const int64_t cap = (int64_t)num_sms * kDriftGridPerSM;
  return (unsigned)(blocks < cap ? (blocks > 0 ? blocks : 1) : cap);
}

void launch_drift_runs(const DriftArgs &a, cudaStream_t s) {
  const DriftK p = make_driftk(a);
  k_drift_runs<<<warp_grid(p.ncells_src, a.num_sms), kDriftWarps * 32, 0, s>>>(p);
}

void launch_drift_spine(const DriftArgs &a, int32_t *rhoc_new, int64_t *rows, int64_t *idx_b_r_new,
                        int64_t *total, cudaStream_t s) {
  const DriftK p = make_driftk(a);
  const Lay &L = *a.L;
  k_ext_counts<<<(unsigned)((p.ncells_src + 255) / 256), 256, 0, s>>>(p, a.phys_count, rhoc_new);
  const int64_t nrows = (int64_t)L.ntile * L.nte * L.nte;
  k_row_sums<<<(unsigned)((nrows + 255) / 256), 256, 0, s>>>(rhoc_new, nrows, L.nte, rows);
  k_scan_rows<<<1, 1024, 0, s>>>(rows, nrows, idx_b_r_new, total);
}

void launch_drift_place(const DriftArgs &a, int32_t nruns, int32_t *scan_tmp, cudaStream_t s) {
  const DriftK p = make_driftk(a);
  const int64_t ndest = (int64_t)a.L->nc * a.L->nc * a.L->nc;
  scan_exclusive_i32(a.dest_runs, ndest, (int32_t *)a.dest_start, scan_tmp, s);
  if (nruns > 0) k_runs_fill<<<(unsigned)((nruns + 255) / 256), 256, 0, s>>>(p, nruns);
  k_runs_order<<<warp_grid(ndest, a.num_sms), kDriftWarps * 32, 0, s>>>(p);
  k_drift_write<<<warp_grid(p.ncells_src, a.num_sms), kDriftWarps * 32, 0, s>>>(p);
  k_halo_fill<<<warp_grid(p.ncells_src, a.num_sms), kDriftWarps * 32, 0, s>>>(p, a.rhoc_new, a.cell_base_new,
                                                                                 a.xp_new, a.vp_new, a.pid_new);
}

void launch_halo_velocities(const Lay &L, const int32_t *rhoc, const int64_t *cell_base, float *vp, int64_t n_used,
                            int num_sms, cudaStream_t s) {
  DriftArgs a{};
  a.L = &L;
  a.nlayer = 1;
  a.n_used = a.n_used_new = n_used;
  const DriftK p = make_driftk(a);
  k_halo_fill<<<warp_grid(p.ncells_src, num_sms), kDriftWarps * 32, 0, s>>>(p, rhoc, cell_base, nullptr, vp,
                                                                              nullptr);
}

}  // namespace cube
