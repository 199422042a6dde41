// Cell-sorted PP binning: a counting sort of every particle of a tile's PP
// region (the tile plus one coarse cell, pp_force_kernel.c:174-180) by PP cell,
// bit-exact with the reference's keys, stable order and cell_start
// (pp_force_kernel.c:196-274).
//
// The input is already sorted by coarse cell (CUBE2's storage order), and a PP
// cell lies inside one coarse cell, so the stable radix sort of the reference
// reduces to a local counting sort per coarse cell: one warp per coarse cell
// histograms its particles over its rcp^3 sub-cells (pass 1), a global
// exclusive scan over all PP cells gives cell_start, and the same warp
// scatters its particles in storage order (pass 2, ranks via __match_any_sync).
// The reference computes keys in float (x = (float)(c + (u+0.5)/2^16),
// floor((float)rcp * x)); the rounding can push a particle into the first PP
// cell of the next coarse cell (|c| >= 128, or rcp not a power of two).  Such
// "spilled" particles are collected in a small list, sorted by (key, storage
// index) and placed ahead of the home particles of their cell, which is where
// the stable sort puts them: every source of a spill precedes the home cell in
// storage order.
//
// Spatial order (used by the kick, not by the parity view): with rcp dividing
// 8, pass 2 can instead order the particles inside each PP cell by the Morton
// index of their 1/8-coarse-cell sub-cell (then storage order).  Keys and
// cell_start are unchanged; the PP work items (chunks of a crowded cell) then
// occupy a compact sub-volume, which lets the PP kernel prune candidates
// against the chunk's bounding box.
#include <cstdio>

#include "common.cuh"

namespace cube {

__global__ void k_cell_table(int64_t nrows, int nte, const int32_t *__restrict__ rhoc,
                             const int64_t *__restrict__ idx_b_r, int64_t *__restrict__ cell_base) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows) return;
  const int32_t *row = rhoc + r * nte;
  int64_t s = idx_b_r[r];
  for (int i = nte - 1; i >= 0; --i) {
    s -= row[i];
    cell_base[r * nte + i] = s;
  }
}

void launch_cell_table(const Lay &L, const int32_t *rhoc, const int64_t *idx_b_r, int64_t *cell_base,
                       cudaStream_t s) {
  int64_t nrows = (int64_t)L.ntile * L.nte * L.nte;
  k_cell_table<<<(unsigned)((nrows + 255) / 256), 256, 0, s>>>(nrows, L.nte, rhoc, idx_b_r, cell_base);
}

struct BinK {
  int nt, ncb, nte, rcs, R, ntile;
  int t_lo, t_n;  // the tiles this launch bins
  int64_t R3;
  int max_rcp3;
  int hist_words;  // shared ints per warp
  int spatial;     // order inside a PP cell by Morton sub-cell (rcp must divide 8)
  int fast;        // every tile-local coarse coordinate lies in [-128, 127]: exact float decode
  const TilePP *tiles;
  const int16_t *xp;
  const int32_t *rhoc;
  const int64_t *cell_base;
  int32_t *count;
  const int32_t *cell_start;
  float4 *spos;
  Spill *spill;
  const int32_t *spill_rank;
  int32_t *spill_n;
  int spill_cap;
  int32_t *err;
};

// number of sorted spill entries with key == g (list sorted by gkey)
__device__ __forceinline__ int spill_count_of(const Spill *sp, int n, int64_t g) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (sp[m].gkey < g) lo = m + 1; else hi = m;
  }
  int a = lo;
  hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (sp[m].gkey <= g) lo = m + 1; else hi = m;
  }
  return lo - a;
}

// decode_pos rounded to float, computed in float: exact (and so equal to the double path) when
// |c| <= 127, since c needs at most 7 integer bits and (u + 0.5) / 2^16 needs 17 fraction bits
__device__ __forceinline__ float decode_pos_f(int c, int16_t xp) {
  return (float)c + ((float)(uint16_t)xp + 0.5f) * (1.0f / 65536.0f);
}

// Morton interleave of up to 2 bits per axis
__device__ __forceinline__ int morton2(int x, int y, int z) {
  auto sp = [](int v) { return (v & 1) | ((v & 2) << 2); };
  return sp(x) | (sp(y) << 1) | (sp(z) << 2);
}

// Pass 1 (SCATTER = false): per-sub-cell counts, spill collection.
// Pass 2 (SCATTER = true): stable placement into spos.
template <bool SCATTER>
__global__ void __launch_bounds__(kWarps * 32) k_pp_bin(BinK p) {
  extern __shared__ int32_t sh_hist[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t wid = (int64_t)blockIdx.x * kWarps + warp;
  if (wid >= (int64_t)p.t_n * p.R3) return;
  // tile and region cell of this warp, in 32-bit arithmetic when the launch's warps fit
  // (64-bit division is a long software sequence)
  int t, cx, cy, cz;
  if ((int64_t)p.t_n * p.R3 <= 0xffffffffLL) {
    const unsigned w = (unsigned)wid, R = (unsigned)p.R, R3 = (unsigned)p.R3;
    const unsigned tq = w / R3, rem = w - tq * R3, q = rem / R, qq = q / R;
    t = p.t_lo + (int)tq;
    cx = (int)(rem - q * R);
    cy = (int)(q - qq * R);
    cz = (int)qq;
  } else {
    t = p.t_lo + (int)(wid / p.R3);
    const int64_t rem = wid - (int64_t)(t - p.t_lo) * p.R3;
    cx = (int)(rem % p.R);
    cy = (int)((rem / p.R) % p.R);
    cz = (int)(rem / ((int64_t)p.R * p.R));
  }
  const TilePP tp = p.tiles[t];
  const int rcp = tp.rcp, S = tp.S, rcp3 = rcp * rcp * rcp;
  int32_t *hist = sh_hist + warp * p.hist_words;
  // extended-tile C index of this region cell and its tile-local coarse coordinate (may be -1 or nt)
  const int ci = p.ncb - 1 + cx, cj = p.ncb - 1 + cy, ck = p.ncb - 1 + cz;
  const int64_t cidx = (((int64_t)t * p.nte + ck) * p.nte + cj) * p.nte + ci;
  const int np = p.rhoc[cidx];
  const int64_t base = p.cell_base[cidx];
  const int lx = cx - 1, ly = cy - 1, lz = cz - 1;
  const int nspill = SCATTER ? min(*p.spill_n, p.spill_cap) : 0;
  // spatial order: bins = (PP sub-cell b, Morton index of the 1/8-coarse-cell sub-cell inside b)
  const bool spatial = SCATTER && p.spatial && (rcp == 2 || rcp == 4);
  const int fs = spatial ? 8 / rcp : 1, s3 = fs * fs * fs;
  const int nbins = rcp3 * s3;
  int32_t *pre = hist + nbins;  // exclusive prefix of the bins (spatial order only)

  // key, spill flag and bin of particle l of this coarse cell (pp_force_kernel.c:213-236)
  auto classify = [&](int l, float &x, float &y, float &z, bool &spilled, bool &bad, int &b, int &bin,
                      int64_t &gkey) {
    const int16_t *q = p.xp + 3 * (base + l);
    // pp_force_kernel.c:213-218: (float)((i-ncb) + ((int16)(xp+ishift)+rshift)*x_resolution)
    if (p.fast) {
      x = decode_pos_f(lx, q[0]);
      y = decode_pos_f(ly, q[1]);
      z = decode_pos_f(lz, q[2]);
    } else {
      x = __double2float_rn(decode_pos(lx, q[0]));
      y = __double2float_rn(decode_pos(ly, q[1]));
      z = __double2float_rn(decode_pos(lz, q[2]));
    }
    // pp_force_kernel.c:226-228: floor(rcp * (x - utile_shift*ntt)) + rcp, float product
    int kx = (int)floorf(__fmul_rn((float)rcp, x)) + rcp;
    int ky = (int)floorf(__fmul_rn((float)rcp, y)) + rcp;
    int kz = (int)floorf(__fmul_rn((float)rcp, z)) + rcp;
    // keys beyond the tile grid (float rounding at the outer halo face) are clamped
    kx = min(max(kx, 0), S - 1);
    ky = min(max(ky, 0), S - 1);
    kz = min(max(kz, 0), S - 1);
    const int rx = kx - rcp * cx, ry = ky - rcp * cy, rz = kz - rcp * cz;
    spilled = (rx >= rcp) | (ry >= rcp) | (rz >= rcp);
    // a key below its own coarse cell cannot come from the float path; reject it
    bad = (rx < 0) | (ry < 0) | (rz < 0) | (rx > rcp) | (ry > rcp) | (rz > rcp);
    b = (rz * rcp + ry) * rcp + rx;
    gkey = tp.cell0 + ((int64_t)kz * S + ky) * S + kx;
    bin = b;
    if (spatial && !spilled && !bad) {
      // 1/8-coarse-cell sub-cell of the same float position, relative to the PP sub-cell
      const int fx = min(max((int)floorf(__fmul_rn(8.f, x)) - 8 * lx, 0), 7);
      const int fy = min(max((int)floorf(__fmul_rn(8.f, y)) - 8 * ly, 0), 7);
      const int fz = min(max((int)floorf(__fmul_rn(8.f, z)) - 8 * lz, 0), 7);
      bin = b * s3 + morton2(fx & (fs - 1), fy & (fs - 1), fz & (fs - 1));  // fs is 2 or 4
    }
  };

  // zero the bins four words at a time (the warp's histogram is 16-byte aligned and at least
  // 1024 words long, so rounding nbins up to a multiple of four stays inside it)
  auto zero_bins = [&]() {
    int4 *h4 = reinterpret_cast<int4 *>(hist);
    for (int q = lane; q < (nbins + 3) / 4; q += 32) h4[q] = make_int4(0, 0, 0, 0);
  };
  zero_bins();
  __syncwarp();

  // Spill-free spatial placement: the histogram pass keeps the bin and float position of its
  // first kCache x 32 particles in registers and the placement pass reuses them, so those
  // particles are classified once (a bad key was already flagged by the counting pass).
  constexpr int kCache = 4;
  int cbin[kCache];
  float cpx[kCache], cpy[kCache], cpz[kCache];
  const bool cached = spatial && nspill == 0;
  if (spatial) {
    // histogram of the bins, then an exclusive prefix per PP sub-cell
    auto hist_one = [&](int l, int &bin_home, float &x, float &y, float &z) {
      bool spilled, bad;
      int b, bin;
      int64_t gkey;
      classify(l, x, y, z, spilled, bad, b, bin, gkey);
      bin_home = -1;
      if (!spilled && !bad) {
        atomicAdd(&hist[bin], 1);
        bin_home = bin;
      }
    };
#pragma unroll
    for (int it = 0; it < kCache; it++) {
      cbin[it] = -1;
      cpx[it] = cpy[it] = cpz[it] = 0.f;
      if (it * 32 + lane < np) hist_one(it * 32 + lane, cbin[it], cpx[it], cpy[it], cpz[it]);
    }
    for (int l = kCache * 32 + lane; l < np; l += 32) {
      int bh;
      float x, y, z;
      hist_one(l, bh, x, y, z);
    }
    __syncwarp();
    // exclusive prefix of the bins inside each PP sub-cell: the 512 bins (rcp^3 sub-cells of
    // s3 bins, rcp 2 or 4) are 16 per lane; s3 = 8 restarts twice inside a lane, s3 = 64 spans
    // four lanes, which a scan over groups of four lanes joins
    {
      const int4 *h4 = reinterpret_cast<const int4 *>(hist) + 4 * lane;
      int4 *p4 = reinterpret_cast<int4 *>(pre) + 4 * lane;
      int v[16];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int4 u = h4[j];
        v[4 * j] = u.x;
        v[4 * j + 1] = u.y;
        v[4 * j + 2] = u.z;
        v[4 * j + 3] = u.w;
      }
      int run = 0;
#pragma unroll
      for (int j = 0; j < 16; j++) {
        if (s3 == 8 && j == 8) run = 0;
        const int c = v[j];
        v[j] = run;
        run += c;
      }
      if (s3 == 64) {
        int incl = run;
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, incl, o, 4);
          if ((lane & 3) >= o) incl += u;
        }
        const int off = incl - run;
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] += off;
      }
#pragma unroll
      for (int j = 0; j < 4; j++) p4[j] = make_int4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
    }
    __syncwarp();
    zero_bins();
    __syncwarp();
  }

  int lstart = 0;
  if (cached) {
    const int bsh = rcp == 2 ? 6 : 3;  // log2 of the bins per PP sub-cell (rcp is 2 or 4)
    const int lr = rcp >> 1;            // log2 rcp
    const int64_t gbase = tp.cell0 + ((int64_t)(rcp * cz) * S + rcp * cy) * S + rcp * cx;
#pragma unroll
    for (int it = 0; it < kCache; it++) {
      if (it * 32 < np) {  // the same for the whole warp
        const int bin = cbin[it];
        const bool home = bin >= 0;
        const unsigned hm = __ballot_sync(0xffffffffu, home);
        int hb = 0, rank = 0;
        unsigned peers = 0;
        if (home) {
          peers = __match_any_sync(hm, bin);
          rank = __popc(peers & ((1u << lane) - 1u));
          hb = hist[bin] + pre[bin];
        }
        __syncwarp();
        if (home) {
          // the PP cell key of the counting pass, from the sub-cell b of this coarse cell
          const int b = bin >> bsh, rx = b & (rcp - 1), ry = (b >> lr) & (rcp - 1), rz = b >> (2 * lr);
          const int64_t gkey = gbase + ((int64_t)rz * S + ry) * S + rx;
          const int64_t pos = (int64_t)p.cell_start[gkey] + hb + rank;
          p.spos[pos] = make_float4(__fmul_rn((float)p.rcs, cpx[it]), __fmul_rn((float)p.rcs, cpy[it]),
                                    __fmul_rn((float)p.rcs, cpz[it]), __int_as_float((int)(base + it * 32 + lane)));
          if (rank == 0) hist[bin] += __popc(peers);
        }
        __syncwarp();
      }
    }
    lstart = kCache * 32;
  }

  for (int l0 = lstart; l0 < np; l0 += 32) {
    const int l = l0 + lane;
    const bool valid = l < np;
    bool spilled = false, bad = false;
    int b = 0, bin = 0;
    int64_t gkey = 0;
    float x = 0.f, y = 0.f, z = 0.f;
    const int64_t ip = base + l;
    if (valid) {
      classify(l, x, y, z, spilled, bad, b, bin, gkey);
      if (bad) atomicOr(p.err, 1 << CUBE_ERR_INVALID);
    }
    const bool home = valid && !spilled && !bad;
    if (!SCATTER) {
      if (home) atomicAdd(&hist[b], 1);
      if (valid && spilled && !bad) {
        int s = atomicAdd(p.spill_n, 1);
        if (s < p.spill_cap) {
          Spill e;
          e.gkey = gkey;
          e.ip = (int32_t)ip;
          e.cell = (int32_t)wid;
          p.spill[s] = e;
        } else {
          atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
        }
      }
    } else {
      const unsigned hm = __ballot_sync(0xffffffffu, home);
      int hb = 0, rank = 0;
      unsigned peers = 0;
      if (home) {
        peers = __match_any_sync(hm, bin);
        rank = __popc(peers & ((1u << lane) - 1u));
        hb = hist[bin] + (spatial ? pre[bin] : 0);
      }
      __syncwarp();
      if (home) {
        int off = 0;
        if (nspill) off = spill_count_of(p.spill, nspill, gkey);
        const int64_t pos = (int64_t)p.cell_start[gkey] + off + hb + rank;
        p.spos[pos] = make_float4(__fmul_rn((float)p.rcs, x), __fmul_rn((float)p.rcs, y),
                                  __fmul_rn((float)p.rcs, z), __int_as_float((int)ip));
        if (rank == 0) hist[bin] += __popc(peers);
      }
      __syncwarp();
    }
  }
  if (!SCATTER) {
    __syncwarp();
    for (int b = lane; b < rcp3; b += 32) {
      const int rx = b % rcp, ry = (b / rcp) % rcp, rz = b / (rcp * rcp);
      const int64_t g = tp.cell0 + ((int64_t)(rcp * cz + rz) * S + (rcp * cy + ry)) * S + (rcp * cx + rx);
      p.count[g] = hist[b];
    }
  }
}

// Sort the spill list by (gkey, ip) in one block, add the spills to the cell
// counts and record each spill's rank inside its cell.
constexpr int kSpillCap = 2048;

__global__ void __launch_bounds__(1024) k_spill_fix(Spill *sp, int32_t *rank, int32_t *spill_n, int cap,
                                                   int32_t *count) {
  __shared__ unsigned long long key[kSpillCap];
  __shared__ int idx[kSpillCap];
  const int n = min(*spill_n, cap);
  if (n == 0) return;
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  for (int i = threadIdx.x; i < np2; i += blockDim.x) {
    key[i] = i < n ? (((unsigned long long)sp[i].gkey << 32) | (unsigned)sp[i].ip) : ~0ull;
    idx[i] = i;
  }
  __syncthreads();
  for (int k = 2; k <= np2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < np2; i += blockDim.x) {
        int l = i ^ j;
        if (l > i) {
          bool up = (i & k) == 0;
          unsigned long long a = key[i], b = key[l];
          if ((a > b) == up) {
            key[i] = b;
            key[l] = a;
            int t = idx[i];
            idx[i] = idx[l];
            idx[l] = t;
          }
        }
      }
      __syncthreads();
    }
  // kSpillCap / 1024 entries per thread: read all, then write back in sorted order
  Spill e[kSpillCap / 1024];
  int m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) e[m++] = sp[idx[i]];
  __syncthreads();
  m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const Spill v = e[m++];
    sp[i] = v;
    int r = 0;
    while (i - r - 1 >= 0 && (long long)(key[i - r - 1] >> 32) == v.gkey) r++;
    rank[i] = r;
    atomicAdd(&count[v.gkey], 1);
  }
}

__global__ void k_spill_place(BinK p) {
  const int n = min(*p.spill_n, p.spill_cap);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Spill e = p.spill[i];
    const int t = (int)(e.cell / p.R3);
    const int64_t rem = e.cell - (int64_t)t * p.R3;
    const int cx = (int)(rem % p.R), cy = (int)((rem / p.R) % p.R), cz = (int)(rem / ((int64_t)p.R * p.R));
    const int16_t *q = p.xp + 3 * (int64_t)e.ip;
    float x = __double2float_rn(decode_pos(cx - 1, q[0]));
    float y = __double2float_rn(decode_pos(cy - 1, q[1]));
    float z = __double2float_rn(decode_pos(cz - 1, q[2]));
    const int64_t pos = (int64_t)p.cell_start[e.gkey] + p.spill_rank[i];
    p.spos[pos] = make_float4(__fmul_rn((float)p.rcs, x), __fmul_rn((float)p.rcs, y), __fmul_rn((float)p.rcs, z),
                              __int_as_float(e.ip));
  }
}

// ---------------------------------------------------------------------------------------------
// exclusive scan of int32 counts -> cell_start (n + 1 entries)

constexpr int kScanThreads = 256, kScanPer = 16, kScanTile = kScanThreads * kScanPer;

size_t scan_tmp_elems(int64_t n) { return (size_t)((n + kScanTile - 1) / kScanTile) + 1; }

__device__ __forceinline__ int block_excl_scan(int v, int *total) {
  __shared__ int ws[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kScanThreads / 32 ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanThreads / 32) ws[lane] = w;
  }
  __syncthreads();
  int incl = x + (warp ? ws[warp - 1] : 0);
  *total = ws[kScanThreads / 32 - 1];
  __syncthreads();
  return incl - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const int32_t *in, int64_t n, int32_t *part) {
  const int64_t b0 = (int64_t)blockIdx.x * kScanTile;
  int s = 0;
  for (int k = 0; k < kScanPer; k++) {
    int64_t i = b0 + (int64_t)k * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  int tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(int32_t *part, int nb, const int32_t *base) {
  int carry = base ? *base : 0;
  for (int c0 = 0; c0 < nb; c0 += kScanThreads) {
    int i = c0 + threadIdx.x;
    int v = i < nb ? part[i] : 0;
    int tot;
    int ex = block_excl_scan(v, &tot);
    if (i < nb) part[i] = ex + carry;
    carry += tot;
  }
  if (threadIdx.x == 0) part[nb] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_down(const int32_t *in, int64_t n, const int32_t *part,
                                                           int nb, int32_t *out) {
  const int64_t b0 = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPer;
  int v[kScanPer];
  int s = 0;
  for (int k = 0; k < kScanPer; k++) {
    int64_t i = b0 + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  int tot;
  int ex = block_excl_scan(s, &tot) + part[blockIdx.x];
  for (int k = 0; k < kScanPer; k++) {
    int64_t i = b0 + k;
    if (i < n) out[i] = ex;
    ex += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = part[nb];
}

void scan_exclusive_i32(const int32_t *in, int64_t n, int32_t *out, int32_t *tmp, cudaStream_t s,
                        const int32_t *base) {
  const int nb = (int)((n + kScanTile - 1) / kScanTile);
  k_scan_reduce<<<nb, kScanThreads, 0, s>>>(in, n, tmp);
  k_scan_top<<<1, kScanThreads, 0, s>>>(tmp, nb, base);
  k_scan_down<<<nb, kScanThreads, 0, s>>>(in, n, tmp, nb, out);
}

static BinK make_bink(const BinArgs &a) {
  const Lay &L = *a.L;
  BinK p;
  p.t_lo = 0;
  p.t_n = L.ntile;
  p.nt = L.nt;
  p.ncb = L.ncb;
  p.nte = L.nte;
  p.rcs = L.rcs;
  p.R = L.nt + 2;
  p.ntile = L.ntile;
  p.R3 = (int64_t)p.R * p.R * p.R;
  p.max_rcp3 = a.max_rcp * a.max_rcp * a.max_rcp;
  p.spatial = a.spatial;
  p.fast = L.nt + 1 <= 127;  // coarse coordinates -1 .. nt
  // histogram words per warp: rcp^3 PP sub-cells, at least 2 x 512 bins for the spatial order
  p.hist_words = p.max_rcp3 < 1024 ? 1024 : p.max_rcp3;
  p.tiles = a.d_tiles;
  p.xp = a.xp;
  p.rhoc = a.rhoc;
  p.cell_base = a.cell_base;
  p.count = a.count;
  p.cell_start = a.cell_start;
  p.spos = a.spos;
  p.spill = a.spill;
  p.spill_rank = a.spill_rank;
  p.spill_n = a.spill_n;
  p.spill_cap = a.spill_cap < kSpillCap ? a.spill_cap : kSpillCap;
  p.err = a.err;
  const size_t shm = sizeof(int32_t) * kWarps * p.hist_words;
  if (shm > 48 * 1024) {  // fine levels (ratio_sf up to 12 or 16) need more than the default window
    cudaFuncSetAttribute(k_pp_bin<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    cudaFuncSetAttribute(k_pp_bin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  }
  return p;
}

void launch_pp_binning(const BinArgs &a, cudaStream_t s) {
  BinK p = make_bink(a);
  const int64_t warps = (int64_t)p.ntile * p.R3;
  const unsigned blocks = (unsigned)((warps + kWarps - 1) / kWarps);
  const size_t shm = sizeof(int32_t) * kWarps * p.hist_words;
  cudaMemsetAsync(a.spill_n, 0, sizeof(int32_t), s);
  k_pp_bin<false><<<blocks, kWarps * 32, shm, s>>>(p);
  k_spill_fix<<<1, 1024, 0, s>>>(a.spill, a.spill_rank, a.spill_n, p.spill_cap, a.count);
  scan_exclusive_i32(a.count, a.ncells, a.cell_start, a.scan_tmp, s);
  k_pp_bin<true><<<blocks, kWarps * 32, shm, s>>>(p);
  k_spill_place<<<8, 256, 0, s>>>(p);
}

bool pp_binning_spill_free(const Lay &L, const TilePP *h_tiles) {
  if (L.nt + 1 > 127) return false;  // the float decode of a coarse coordinate is exact up to 127
  for (int t = 0; t < L.ntile; t++)
    if (h_tiles[t].rcp & (h_tiles[t].rcp - 1)) return false;  // rcp * x exact for powers of two
  return true;
}

void launch_pp_binning_tiles(const BinArgs &a, const TilePP *h_tiles, int t_lo, int t_hi, cudaStream_t s) {
  BinK p = make_bink(a);
  p.t_lo = t_lo;
  p.t_n = t_hi - t_lo;
  const int64_t warps = (int64_t)p.t_n * p.R3;
  const unsigned blocks = (unsigned)((warps + kWarps - 1) / kWarps);
  const size_t shm = sizeof(int32_t) * kWarps * p.hist_words;
  if (t_lo == 0) cudaMemsetAsync(a.spill_n, 0, sizeof(int32_t), s);
  k_pp_bin<false><<<blocks, kWarps * 32, shm, s>>>(p);
  // the tiles' PP cells are consecutive; their cell starts continue from the previous tiles'
  // total, which those tiles' scan left at cell_start[cell0]
  const int64_t c0 = h_tiles[t_lo].cell0;
  const TilePP &tl = h_tiles[t_hi - 1];
  const int64_t nc = tl.cell0 + (int64_t)tl.S * tl.S * tl.S - c0;
  scan_exclusive_i32(a.count + c0, nc, a.cell_start + c0, a.scan_tmp, s, t_lo ? a.cell_start + c0 : nullptr);
  k_pp_bin<true><<<blocks, kWarps * 32, shm, s>>>(p);
}

size_t bin_smem_bytes(int max_rcp) {
  const int r3 = max_rcp * max_rcp * max_rcp;
  return sizeof(int32_t) * kWarps * (r3 < 1024 ? 1024 : r3);
}

}  // namespace cube
