// PP short-range pair force over the neighbouring PP cells
// (pp_force_kernel.c:282-325, pp_force_kernel.cu:192-250) and the kick of the
// interior particles (pp_force_kernel.c:339-364).
//
// Work decomposition.  An item is one interior PP cell, or a 32-particle chunk
// of a crowded one.  A particle of range rc needs the cells within
// R = ceil(rc * rcp / ratio_cs) of its own (pp_force_kernel.cu:205); the rows
// (dy, dz) of that stencil whose nearest point is farther than rc are skipped,
// and the cells of a row are one contiguous range of the cell-sorted array.
// Items are bucketed by cost (log2 of candidates per lane group) and a
// persistent kernel hands them out heaviest first through an atomic queue
// head, so the lognormal occupancy of clustered boxes does not leave a tail.
//
// Inside an item one warp splits its 32 lanes into floor(32/ni) groups of ni
// lanes; lane (group g, particle i) walks every ngrp-th candidate.  Candidates
// are staged per warp in shared memory (coalesced float4 loads, broadcast
// reads).  Only about 15% of the stencil candidates lie inside the cutoff, so
// evaluating the pair law for every candidate would spend most issue slots on
// rejected pairs: instead each lane pushes its accepted (dx, dy, dz, r^2)
// into its own shared-memory queue, and when any lane's queue is full the
// warp drains all queues in lock-step rounds.  The pair law is evaluated
// without divisions or branches (one rsqrt and a degree-6 Horner polynomial
// with per-lane coefficient selection).  Each lane keeps Kahan-compensated
// sums updated once per drain; the groups of a particle are merged with warp
// shuffles (TwoSum), and the owning lane applies af*mass^2, the kick, f2max
// and vmax.
#include "common.cuh"

namespace cube {

constexpr int kPPThreads = 256;
constexpr int kPPWarps = kPPThreads / 32;
constexpr int kJTile = 128;  // staged candidates per warp
constexpr int kBuckets = 32;
constexpr size_t kPPSmem = sizeof(float4) * kPPWarps * kJTile;

// basic_functions.f08:95-109 / pp_force_kernel.c:45-74 in FP32, same operation order
__device__ __forceinline__ float F_ra(float r, float apm) {
  float ep = 2.0f * r / apm;
  if (apm == 0.0f || ep > 2.0f) return 1.0f / (r * r);
  if (ep > 1.0f) {
    float ep2 = ep * ep, ep3 = ep2 * ep, ep4 = ep3 * ep, ep5 = ep4 * ep, ep6 = ep5 * ep;
    return (1.0f / 35.0f / (apm * apm)) *
           (12.0f / ep2 - 224.0f + 896.0f * ep - 840.0f * ep2 + 224.0f * ep3 + 70.0f * ep4 - 48.0f * ep5 +
            7.0f * ep6);
  }
  if (ep > 0.0f) {
    float ep3 = ep * ep * ep, ep4 = ep3 * ep, ep5 = ep4 * ep, ep6 = ep5 * ep;
    return (1.0f / 35.0f / (apm * apm)) * (224.0f * ep - 224.0f * ep3 + 70.0f * ep4 + 48.0f * ep5 - 21.0f * ep6);
  }
  return 0.0f;
}

// F_ra(r,app) - F_ra(r,rc) for 0 < r < rc, as a function of r^2, with per-cell constants and
// no division: for r > app it equals A/r^2 - sum_k c_k ep^k with ep = 2r/rc, where
//   outer (ep > 1): A = 32/35 (the 12/ep^2 term folded in), c = [-224,896,-840,224,70,-48,7]/(35 rc^2)
//   inner:          A = 1,                                  c = [0,224,0,-224,70,48,-21]/(35 rc^2)
// Returns the scale s such that the pair force is s * (dx, dy, dz).
struct PairLaw {
  float cep, app2, app, rc;
  float o0, o1, o2, o3, o4, o5, o6, n1, n3, n4, n5, n6;
  __device__ __forceinline__ void init(float rc_, float app_) {
    rc = rc_;
    app = app_;
    const float k35 = 1.0f / (35.0f * rc_ * rc_);
    cep = 2.0f / rc_;
    app2 = app_ * app_;
    o0 = -224.f * k35, o1 = 896.f * k35, o2 = -840.f * k35, o3 = 224.f * k35, o4 = 70.f * k35, o5 = -48.f * k35,
    o6 = 7.f * k35;
    n1 = 224.f * k35, n3 = -224.f * k35, n4 = 70.f * k35, n5 = 48.f * k35, n6 = -21.f * k35;
  }
  __device__ __forceinline__ float scale(float r2) const {
    const float invr = rsqrtf(r2);
    const float ir2 = invr * invr;
    const float ep = r2 * invr * cep;
    const bool outer = ep > 1.0f;
    float q = outer ? o6 : n6;
    q = fmaf(q, ep, outer ? o5 : n5);
    q = fmaf(q, ep, outer ? o4 : n4);
    q = fmaf(q, ep, outer ? o3 : n3);
    q = fmaf(q, ep, outer ? o2 : 0.0f);
    q = fmaf(q, ep, outer ? o1 : n1);
    q = fmaf(q, ep, outer ? o0 : 0.0f);
    float fpp = fmaf(outer ? (32.0f / 35.0f) : 1.0f, ir2, -q);
    if (r2 <= app2) {  // inside the softening length: the exact S2 law (rare)
      const float r = r2 * invr;
      fpp = F_ra(r, app) - F_ra(r, rc);
    }
    return fpp * invr;
  }
};

__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float x) {
  float y = x - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}

// (hi, lo) + (hi2, lo2) with an error-free TwoSum of the high parts
__device__ __forceinline__ void two_sum_merge(float &hi, float &lo, float hi2, float lo2) {
  float s = hi + hi2;
  float bp = s - hi;
  float err = (hi - (s - bp)) + (hi2 - bp);
  hi = s;
  lo = lo + lo2 + err;
}

struct PPK {
  int nt, ntt, nns, nnt, ntile, rcs;
  const TilePP *tiles;
  const int32_t *cs;
  const float4 *spos;
  const float *range_loc;
  int4 *items;
  int32_t *bucket;  // [0,32) counts, [32,64) cursors
  int32_t *head;
  int64_t item_cap;
  float *vp;
  float mass2, kick, app;
  float *out;
  int want_vmax;
  int32_t *err;
  int64_t max_cells;          // max interior PP cells per tile (grid sizing)
  unsigned long long *pairs;  // COUNT mode: accepted ordered pairs
};

// PP range of the particles of interior cell (x, y, z) of tile t (per subtile, pp_force_kernel.cu:776-790)
__device__ __forceinline__ float cell_range(const PPK &p, int t, int x, int y, int z, int rcp) {
  const int tx = t % p.nnt, ty = (t / p.nnt) % p.nnt, tz = t / (p.nnt * p.nnt);
  const int sx = (x / rcp - 1) / p.ntt, sy = (y / rcp - 1) / p.ntt, sz = (z / rcp - 1) / p.ntt;
  return p.range_loc[(((tz * p.nnt + ty) * p.nnt + tx) * p.nns + sz) * p.nns * p.nns + sy * p.nns + sx];
}

// stencil radius in cells and the row test: row (dy, dz) can hold a particle within rc
__device__ __forceinline__ int stencil_radius(float rc, int rcp, int rcs) {
  return (int)ceilf(rc * (float)rcp / (float)rcs);
}
__device__ __forceinline__ bool row_needed(int dy, int dz, float h, float rc2) {
  const float ay = (float)max(abs(dy) - 1, 0) * h, az = (float)max(abs(dz) - 1, 0) * h;
  return ay * ay + az * az < rc2;
}

// cost bucket of a chunk with ni i-particles and nj candidates, heavy = high index:
// the warp walks the candidates in floor(32/ni) lane groups
__device__ __forceinline__ int cost_bucket(int ni, int64_t nj) {
  int64_t c = nj / (32 / max(ni, 1));
  if (c < 1) c = 1;
  int b = 63 - __clzll(c);
  return b > kBuckets - 1 ? kBuckets - 1 : b;
}

// Enumerate interior PP cells; pass 0 counts items per bucket, pass 1 emits them.
template <int PASS>
__global__ void __launch_bounds__(256) k_pp_items(PPK p) {
  __shared__ int sc[kBuckets], sbase[kBuckets], soff[kBuckets];
  if (threadIdx.x < kBuckets) sc[threadIdx.x] = 0;
  if (PASS == 1 && threadIdx.x == 0) {
    int acc = 0;
    for (int b = kBuckets - 1; b >= 0; --b) {
      soff[b] = acc;
      acc += p.bucket[b];
    }
  }
  __syncthreads();
  const int t = blockIdx.y;
  const TilePP tp = p.tiles[t];
  const int rcp = tp.rcp, S = tp.S, npg = p.nt * rcp;
  const int64_t ncell = (int64_t)npg * npg * npg;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int nchunks = 0, ni = 0;
  int64_t nj = 0, g = 0;
  if (c < ncell) {
    const int x = (int)(c % npg) + rcp, y = (int)((c / npg) % npg) + rcp, z = (int)(c / ((int64_t)npg * npg)) + rcp;
    g = tp.cell0 + ((int64_t)z * S + y) * S + x;
    ni = p.cs[g + 1] - p.cs[g];
    if (ni > 0) {
      const float rc = cell_range(p, t, x, y, z, rcp);
      const int R = stencil_radius(rc, rcp, p.rcs);
      if (R > rcp) atomicOr(p.err, 1 << CUBE_ERR_INVALID);  // beyond the one coarse-cell halo
      const float h = (float)p.rcs / (float)rcp;
      const int Rc = min(R, rcp);
      for (int dz = -Rc; dz <= Rc; dz++)
        for (int dy = -Rc; dy <= Rc; dy++) {
          if (!row_needed(dy, dz, h, rc * rc)) continue;
          const int64_t b = g + ((int64_t)dz * S + dy) * S;
          nj += p.cs[b + Rc + 1] - p.cs[b - Rc];
        }
      nchunks = (ni + 31) >> 5;
    }
  }
  int myrank[4];
  int mybucket[4];
  // chunks beyond the first few per thread are rare; handle the first 4 with local ranks,
  // the rest with direct global atomics
  for (int k = 0; k < nchunks; k++) {
    const int nik = min(32, ni - 32 * k);
    const int b = cost_bucket(nik, nj);
    if (k < 4) {
      mybucket[k] = b;
      myrank[k] = atomicAdd(&sc[b], 1);
    } else if (PASS == 0) {
      atomicAdd(&p.bucket[b], 1);
    } else {
      const int slot = soff[b] + atomicAdd(&p.bucket[kBuckets + b], 1);
      if (slot < p.item_cap) p.items[slot] = make_int4((int)g, k, t, 0);
      else atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
    }
  }
  __syncthreads();
  if (threadIdx.x < kBuckets) {
    const int n = sc[threadIdx.x];
    if (PASS == 0) {
      if (n) atomicAdd(&p.bucket[threadIdx.x], n);
    } else {
      sbase[threadIdx.x] = n ? atomicAdd(&p.bucket[kBuckets + threadIdx.x], n) : 0;
    }
  }
  if (PASS == 1) {
    __syncthreads();
    for (int k = 0; k < nchunks && k < 4; k++) {
      const int b = mybucket[k];
      const int64_t slot = (int64_t)soff[b] + sbase[b] + myrank[k];
      if (slot < p.item_cap) p.items[slot] = make_int4((int)g, k, t, 0);
      else atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
    }
  }
}

// COUNT = false: forces and kick.  COUNT = true: only count the accepted ordered
// pairs 0 < r^2 < rc^2 (the algorithmic work of the kick, for the roofline).
template <bool COUNT>
__global__ void __launch_bounds__(kPPThreads, 3) k_pp_force(PPK p) {
  extern __shared__ float4 pp_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float4 *buf = pp_smem + warp * kJTile;
  int total = 0;
  {
    int v = lane < kBuckets ? p.bucket[lane] : 0;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    total = min((int64_t)v, p.item_cap);
  }
  float f2w = 0.f, vm0 = 0.f, vm1 = 0.f, vm2 = 0.f;
  unsigned long long npairs = 0;
  for (;;) {
    int it = 0;
    if (lane == 0) it = atomicAdd(p.head, 1);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= total) break;
    const int4 item = p.items[it];
    const int64_t g = (int64_t)(unsigned)item.x;
    const int t = item.z;
    const TilePP tp = p.tiles[t];
    const int S = tp.S, rcp = tp.rcp;
    const int64_t loc = g - tp.cell0;
    const int x = (int)(loc % S), y = (int)((loc / S) % S), z = (int)(loc / ((int64_t)S * S));
    const float rc = cell_range(p, t, x, y, z, rcp);
    const float rc2 = rc * rc;
    const int R = min(stencil_radius(rc, rcp, p.rcs), rcp);
    const float h = (float)p.rcs / (float)rcp;
    PairLaw law;
    law.init(rc, p.app);

    const int i0 = p.cs[g] + item.y * 32;
    const int ni = min(32, p.cs[g + 1] - i0);
    // lanes = ngrp groups of ni lanes; group `grp` walks every ngrp-th candidate
    const int ngrp = 32 / ni;
    const int il = lane % ni, grp = lane / ni;
    const bool has_i = grp < ngrp;  // the 32 mod ni leftover lanes idle
    const float4 pi = p.spos[i0 + il];

    // bounding box of the item's particles: candidates farther than rc from it are dropped
    // while staging, so the pair loop below only sees possibly-interacting candidates
    const float blx = warp_min(pi.x), bhx = warp_max(pi.x), bly = warp_min(pi.y), bhy = warp_max(pi.y),
                blz = warp_min(pi.z), bhz = warp_max(pi.z);
    float sx_ = 0.f, cx_ = 0.f, sy_ = 0.f, cy_ = 0.f, sz_ = 0.f, cz_ = 0.f;
    int nbuf = 0;  // staged candidates (warp-uniform)
    auto flush = [&]() {
      __syncwarp();
      float px = 0.f, py = 0.f, pz = 0.f;
#pragma unroll 4
      for (int q = has_i ? grp : nbuf; q < nbuf; q += ngrp) {
        const float4 pj = buf[q];
        const float dx = pj.x - pi.x, dy_ = pj.y - pi.y, dz_ = pj.z - pi.z;
        const float r2 = dx * dx + dy_ * dy_ + dz_ * dz_;
        const bool ok = (r2 > 0.0f) & (r2 < rc2);
        if (COUNT) {
          npairs += ok ? 1ull : 0ull;
        } else {
          // evaluated for every candidate and masked: a divergent accept branch would
          // run on nearly every iteration of a 32-lane warp anyway
          const float s = ok ? law.scale(r2) : 0.0f;
          px = fmaf(s, dx, px);
          py = fmaf(s, dy_, py);
          pz = fmaf(s, dz_, pz);
        }
      }
      if (!COUNT) {
        kahan_add(sx_, cx_, px);
        kahan_add(sy_, cy_, py);
        kahan_add(sz_, cz_, pz);
      }
      nbuf = 0;
      __syncwarp();
    };
    for (int dz = -R; dz <= R; dz++)
      for (int dy = -R; dy <= R; dy++) {
        if (!row_needed(dy, dz, h, rc2)) continue;
        const int64_t b = g + ((int64_t)dz * S + dy) * S;
        const int js = p.cs[b - R], je = p.cs[b + R + 1];
        for (int jb = js; jb < je; jb += 32) {
          const int q = jb + lane;
          bool keep = q < je;
          float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
          if (keep) {
            pj = p.spos[q];
            const float ex = fmaxf(fmaxf(blx - pj.x, pj.x - bhx), 0.f);
            const float ey = fmaxf(fmaxf(bly - pj.y, pj.y - bhy), 0.f);
            const float ez = fmaxf(fmaxf(blz - pj.z, pj.z - bhz), 0.f);
            keep = ex * ex + ey * ey + ez * ez < rc2;
          }
          const unsigned m = __ballot_sync(0xffffffffu, keep);
          if (keep) buf[nbuf + __popc(m & ((1u << lane) - 1u))] = pj;
          nbuf += __popc(m);
          if (nbuf > kJTile - 32) flush();
        }
      }
    if (nbuf) flush();
    // merge the lane groups of each i-particle (tree over groups, stride s*ni lanes);
    // Kahan c is the negated low part
    float hx = sx_, lx = -cx_, hy = sy_, ly = -cy_, hz = sz_, lz = -cz_;
    for (int s = 1; s < ngrp; s <<= 1) {
      const int delta = s * ni;
      const float ohx = __shfl_down_sync(0xffffffffu, hx, delta), olx = __shfl_down_sync(0xffffffffu, lx, delta);
      const float ohy = __shfl_down_sync(0xffffffffu, hy, delta), oly = __shfl_down_sync(0xffffffffu, ly, delta);
      const float ohz = __shfl_down_sync(0xffffffffu, hz, delta), olz = __shfl_down_sync(0xffffffffu, lz, delta);
      if ((grp % (2 * s)) == 0 && grp + s < ngrp) {
        two_sum_merge(hx, lx, ohx, olx);
        two_sum_merge(hy, ly, ohy, oly);
        two_sum_merge(hz, lz, ohz, olz);
      }
    }
    if (!COUNT && grp == 0 && has_i) {
      const float ax = (hx + lx) * p.mass2, ay = (hy + ly) * p.mass2, az = (hz + lz) * p.mass2;
      f2w = fmaxf(f2w, ax * ax + ay * ay + az * az);
      const int64_t ip = (int64_t)__float_as_int(pi.w);
      float *v = p.vp + 3 * ip;
      const float v0 = v[0] + ax * p.kick, v1 = v[1] + ay * p.kick, v2 = v[2] + az * p.kick;
      v[0] = v0;
      v[1] = v1;
      v[2] = v2;
      vm0 = fmaxf(vm0, fabsf(v0));
      vm1 = fmaxf(vm1, fabsf(v1));
      vm2 = fmaxf(vm2, fabsf(v2));
    }
  }
  if (COUNT) {
    for (int o = 16; o; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if (lane == 0) atomicAdd(p.pairs, npairs);
    return;
  }
  f2w = warp_max(f2w);
  if (lane == 0) atomic_max_nonneg(&p.out[1], f2w);
  if (p.want_vmax) {
    vm0 = warp_max(vm0);
    vm1 = warp_max(vm1);
    vm2 = warp_max(vm2);
    if (lane == 0) {
      atomic_max_nonneg(&p.out[2], vm0);
      atomic_max_nonneg(&p.out[3], vm1);
      atomic_max_nonneg(&p.out[4], vm2);
    }
  }
}

static PPK make_ppk(const PPArgs &a) {
  const Lay &L = *a.L;
  PPK p;
  p.nt = L.nt;
  p.ntt = L.ntt;
  p.nns = L.nns;
  p.nnt = L.nnt;
  p.ntile = L.ntile;
  p.rcs = L.rcs;
  p.tiles = a.d_tiles;
  p.cs = a.cell_start;
  p.spos = a.spos;
  p.range_loc = a.range_loc;
  p.items = a.items;
  p.bucket = a.bucket;
  p.head = a.head;
  p.item_cap = a.item_cap;
  p.vp = a.vp;
  p.mass2 = a.mass2;
  p.kick = a.kick;
  p.app = L.app;
  p.out = a.out;
  p.want_vmax = a.want_vmax;
  p.err = a.err;
  p.pairs = a.pairs;
  int max_rcp = 1;
  for (int t = 0; t < L.ntile; t++) max_rcp = a.h_tiles[t].rcp > max_rcp ? a.h_tiles[t].rcp : max_rcp;
  const int64_t npg = (int64_t)L.nt * max_rcp;
  p.max_cells = npg * npg * npg;
  return p;
}

void launch_pp_items(const PPArgs &a, cudaStream_t s) {
  PPK p = make_ppk(a);
  cudaMemsetAsync(a.bucket, 0, sizeof(int32_t) * 2 * kBuckets, s);
  dim3 grid((unsigned)((p.max_cells + 255) / 256), (unsigned)a.L->ntile);
  k_pp_items<0><<<grid, 256, 0, s>>>(p);
  k_pp_items<1><<<grid, 256, 0, s>>>(p);
}

// one persistent block per resident slot: blocks beyond the resident count would
// only start once the queue is empty
static int resident_blocks(const void *fn, int num_sms) {
  static int cached[2] = {0, 0};
  const int which = fn == (const void *)k_pp_force<true> ? 1 : 0;
  if (!cached[which]) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPPSmem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPPThreads, kPPSmem);
    cached[which] = per_sm > 0 ? per_sm : 1;
  }
  return cached[which] * num_sms;
}

void launch_pp_force(const PPArgs &a, cudaStream_t s) {
  PPK p = make_ppk(a);
  cudaMemsetAsync(a.head, 0, sizeof(int32_t), s);
  if (a.pairs) {
    const void *fn = (const void *)k_pp_force<true>;
    k_pp_force<true><<<resident_blocks(fn, a.num_sms), kPPThreads, kPPSmem, s>>>(p);
  } else {
    const void *fn = (const void *)k_pp_force<false>;
    k_pp_force<false><<<resident_blocks(fn, a.num_sms), kPPThreads, kPPSmem, s>>>(p);
  }
}

}  // namespace cube
