// PP short-range pair force over the neighbouring PP cells
// (pp_force_kernel.c:282-325, pp_force_kernel.cu:192-250) and the kick of the
// interior particles (pp_force_kernel.c:339-364).
//
// Work decomposition.  An item is one interior PP cell, or a C-particle
// chunk of a crowded one (the kick's binning orders a cell's particles by
// Morton sub-cell, so a chunk occupies a compact sub-volume).  A particle of
// range rc needs the cells within R = ceil(rc * rcp / ratio_cs) of its own
// (pp_force_kernel.cu:205); the rows (dy, dz) of that stencil whose nearest
// point is farther than rc are skipped, and the cells of a row are one
// contiguous range of the cell-sorted array.  Items are bucketed by cost
// (log2 of candidates per lane group) and a persistent kernel hands them out
// heaviest first through an atomic queue head, so the lognormal occupancy of
// clustered boxes does not leave a tail.
//
// Inside an item one warp splits its 32 lanes into floor(32/ni) groups of ni
// lanes; lane (group g, particle i) walks every ngrp-th staged candidate.  The
// needed rows are laid end to end in a per-warp row table, so every staging
// step loads 32 candidates (prefetched one step ahead) however short the rows
// are.  A candidate is staged in shared memory only if it lies within rc of
// the bounding box of the item's particles, which removes most of the stencil
// volume before the pair law runs.  The pair law is evaluated without
// divisions or selects: the inner piece of the S2 law differs from the outer
// one by (1 - ep)^6 (12 + 72 ep + 28 ep^2) / ep^2, so one Horner polynomial in
// r plus max(1 - ep, 0)^6 times a quadratic covers both.  Each lane keeps
// Kahan-compensated sums updated once per flush of the staging buffer; the
// groups of a particle are merged with warp shuffles (TwoSum), and the owning
// lane applies af*mass^2, the kick, f2max and vmax.
//
// Packed shapes evaluate the pair law on sm_100's f32x2 arithmetic (FFMA2, FMUL2, FADD2):
// a lane takes two staged candidates per round, which halves the issue slots of the law;
// every operation rounds as its scalar form, so each pair's force is bit for bit the scalar
// one and only the summation order differs.  The kernel is issue-bound, so the per-lane state
// that is touched once per flush or item (Kahan sums, maxima, the owned particle's velocity,
// which a cp.async brings in while the item runs) lives in shared memory, and a warp pops
// its work items four at a time, each carrying its first particle, count, stencil radius
// and pair-law constants (k_pp_items computes them once per kick).
#include <type_traits>
#include <utility>

#include "common.cuh"

namespace cube {

constexpr int kPPThreads = 256;
constexpr int kPPWarps = kPPThreads / 32;
constexpr int kMaxRows = 96;  // stencil rows per row table (a multiple of 32)
constexpr int kBuckets = 32;

// Kernel shapes the autotuner picks from (the host times each on the kick's own particles):
// chunk = i-particles per work item, so a crowded PP cell of n particles gets ceil(n / chunk)
// warps; jtile = candidates a warp stages in shared memory between two flushes; unroll = unroll
// factor of the pair loop; blocks = resident blocks per SM the registers are budgeted for
// (4: 64 registers a thread, 3: 80), packed = pair law on f32x2 arithmetic.  Shape 0 is the
// default; the last shape is the scalar form, kept for comparison.
constexpr PPShapeDesc kShapes[] = {
    {16, 128, 2, 4, 1}, {16, 128, 1, 4, 1}, {16, 256, 2, 4, 1}, {16, 128, 4, 4, 1}, {16, 64, 2, 4, 1},
    {16, 128, 2, 3, 1}, {16, 256, 1, 4, 1}, {8, 256, 1, 4, 1},  {8, 256, 2, 4, 1},  {16, 128, 8, 4, 1},
    {32, 128, 2, 4, 1}, {16, 256, 4, 4, 1}, {16, 96, 4, 4, 1},  {16, 64, 4, 4, 1},  {16, 64, 1, 4, 1},
    {16, 64, 2, 4, 0}};
// the pair-count kernel (scalar loop, the work list of shape 0)
constexpr PPShapeDesc kCountShape = {kShapes[0].chunk, 64, 2, 4, 0};
constexpr int kNumShapes = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
static_assert(kNumShapes <= kMaxPPShapes, "shape table");
constexpr int min_shape_chunk() {
  int c = kShapes[0].chunk;
  for (int i = 1; i < kNumShapes; i++) c = kShapes[i].chunk < c ? kShapes[i].chunk : c;
  return c;
}
constexpr int kMinChunk = min_shape_chunk();  // the work list capacity is sized for it
static_assert(kShapes[0].chunk == kPPChunk, "shape 0 is the default shape");
// per-warp shared memory: the staged candidates (scalar: float4 [jtile + 32]; packed: x, y and z
// planes of jtile + 64 floats each), then the row table
constexpr size_t pp_stage_bytes(int jtile, bool packed) {
  return packed ? 3 * sizeof(float) * (jtile + 64) : sizeof(float4) * (jtile + 32);
}
// per-lane state kept in shared memory rather than registers (it is touched once per flush or
// item): Kahan sums and compensations of x, y, z, f2 and |v| maxima, the owned particle's
// velocity (copied in asynchronously when the item starts); then the item's bounding box and
// the row-table cache, then the batch of work items the warp popped
constexpr int kLaneFields = 13;
constexpr int kPop = 4;  // work items a warp takes from the queue at a time
constexpr size_t pp_state_bytes() { return sizeof(float) * (kLaneFields * 32 + 8) + sizeof(PPItem) * kPop; }
constexpr size_t pp_smem_warp(int jtile, bool packed) {
  return pp_stage_bytes(jtile, packed) + sizeof(int2) * kMaxRows + pp_state_bytes();
}
constexpr size_t pp_smem_block(int jtile, bool packed) { return pp_smem_warp(jtile, packed) * kPPWarps; }
constexpr bool pp_smem_aligned() {
  for (int jt = 32; jt <= 256; jt += 32)
    if (pp_smem_warp(jt, false) % 16 || pp_smem_warp(jt, true) % 16 || pp_stage_bytes(jt, true) % 16) return false;
  return true;
}
static_assert(pp_smem_aligned() && (sizeof(int2) * kMaxRows + sizeof(float) * 32 * kLaneFields) % 16 == 0,
              "16-byte aligned warp areas, bounding box and item batch");

// F_ra(r, apm) of basic_functions.f08:95-109 / pp_force_kernel.c:45-74 in FP32 without
// divisions or branches: with ep = 2r/apm = r * ce and k = (1/35) / apm^2,
//   ep <= 1: k (224ep - 224ep^3 + 70ep^4 + 48ep^5 - 21ep^6)
//   ep > 1:  k (12/ep^2 - 224 + 896ep - 840ep^2 + 224ep^3 + 70ep^4 - 48ep^5 + 7ep^6)
//            = (3/35)/r^2 + k (-224 + 896ep - ... + 7ep^6)      (k 12/ep^2 = (3/35)/r^2)
//   ep > 2:  1/r^2
__device__ __forceinline__ float F_ra_soft(float r, float ir2, float ce, float k) {
  const float ep = r * ce;
  float qo = fmaf(7.0f, ep, -48.0f);
  qo = fmaf(qo, ep, 70.0f);
  qo = fmaf(qo, ep, 224.0f);
  qo = fmaf(qo, ep, -840.0f);
  qo = fmaf(qo, ep, 896.0f);
  qo = fmaf(qo, ep, -224.0f);
  float qi = fmaf(-21.0f, ep, 48.0f);
  qi = fmaf(qi, ep, 70.0f);
  qi = fmaf(qi, ep, -224.0f);
  qi = qi * ep;
  qi = fmaf(qi, ep, 224.0f);
  qi = qi * ep;
  return ep > 2.0f ? ir2 : (ep > 1.0f ? fmaf(k, qo, (3.0f / 35.0f) * ir2) : k * qi);
}

// 1/sqrt(x) on the special-function unit with subnormal inputs flushed (rsqrt.approx.ftz):
// squared pair distances are either 0 (masked), at least (2^-16 fine cell)^2 or a far sentinel,
// never subnormal, so only rsqrtf's handling of subnormal inputs is left out
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// packed f32x2 arithmetic (sm_100: one instruction updates both halves, each rounded as the
// scalar operation)
__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// s(r^2) = (F_ra(r,app) - F_ra(r,rc)) / r for 0 <= r < rc, so that the pair force is s * (dx, dy, dz).
// With ep = 2r/rc and k = 1/(35 rc^2), for r > app:
//   outer (ep > 1): 1/r^2 - F_ra(r,rc) = (32/35)/r^2 - k P(ep),  P = -224 + 896ep - 840ep^2 + 224ep^3
//                                                                     + 70ep^4 - 48ep^5 + 7ep^6
//   inner (ep <= 1): the outer form plus k (1-ep)^6 (12 + 72ep + 28ep^2) / ep^2
//                    = (1/r^2) (1-ep)^6 (3/35 + 18/35 ep + 7/35 ep^2)
// (expanding the product gives back the inner polynomial 224ep - 224ep^3 + 70ep^4 + 48ep^5 - 21ep^6).
// The polynomial coefficients are literals (instruction immediates), so a law costs two registers
// per item (2/rc and 1/(35 rc^2)).  Inside the softening length (soft(), a second pass over
// the pairs the main loop flags) both F_ra terms are evaluated directly.
struct PairLaw {
  float cep, k35;
  // the constants of range rc, as k_pp_items stores them in the work item
  __device__ __forceinline__ static float k35_of(float rc_) { return 1.0f / (35.0f * rc_ * rc_); }
  __device__ __forceinline__ static float cep_of(float rc_) { return 2.0f / rc_; }
  __device__ __forceinline__ void init(const PPItem &it) {
    k35 = it.k35;
    cep = it.cep;
  }
  __device__ __forceinline__ float scale(float r2) const {
    const float invr = rsqrt_ftz(r2);
    const float ir2 = invr * invr;
    const float ep = r2 * invr * cep;
    float q = fmaf(7.0f, ep, -48.0f);
    q = fmaf(q, ep, 70.0f);
    q = fmaf(q, ep, 224.0f);
    q = fmaf(q, ep, -840.0f);
    q = fmaf(q, ep, 896.0f);
    q = fmaf(q, ep, -224.0f);
    const float u = fmaxf(1.0f - ep, 0.0f);
    const float u2 = u * u;
    const float u6 = u2 * u2 * u2;
    const float w = fmaf(fmaf(7.0f / 35.0f, ep, 18.0f / 35.0f), ep, 3.0f / 35.0f);
    const float br = fmaf(u6, w, 32.0f / 35.0f);
    return fmaf(br, ir2, -q * k35) * invr;
  }
  // scale() of two squared distances on packed f32x2 arithmetic: every operation is the scalar
  // one, rounded the same way, so each half equals scale() of that half bit for bit
  __device__ __forceinline__ float2 scale2(float2 r2) const {
    const float2 invr = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    const float2 ir2 = mul2(invr, invr);
    const float2 ep = mul2(mul2(r2, invr), dup(cep));
    float2 q = fma2(dup(7.0f), ep, dup(-48.0f));
    q = fma2(q, ep, dup(70.0f));
    q = fma2(q, ep, dup(224.0f));
    q = fma2(q, ep, dup(-840.0f));
    q = fma2(q, ep, dup(896.0f));
    q = fma2(q, ep, dup(-224.0f));
    float2 u = fma2(ep, dup(-1.0f), dup(1.0f));
    u = make_float2(fmaxf(u.x, 0.0f), fmaxf(u.y, 0.0f));
    const float2 u2 = mul2(u, u);
    const float2 u6 = mul2(mul2(u2, u2), u2);
    const float2 w = fma2(fma2(dup(7.0f / 35.0f), ep, dup(18.0f / 35.0f)), ep, dup(3.0f / 35.0f));
    const float2 br = fma2(u6, w, dup(32.0f / 35.0f));
    return mul2(fma2(br, ir2, mul2(q, dup(-k35))), invr);
  }
  // 0 < r <= app: (F_ra(r, app) - F_ra(r, rc)) / r; cea = 2/app, ka = (1/35)/app^2
  __device__ __forceinline__ float soft(float r2, float cea, float ka) const {
    const float invr = rsqrt_ftz(r2);
    const float r = r2 * invr, ir2 = invr * invr;
    return (F_ra_soft(r, ir2, cea, ka) - F_ra_soft(r, ir2, cep, k35)) * invr;
  }
};

// order-preserving map between floats and ints, for the integer warp reductions (redux.sync)
__device__ __forceinline__ int float_key(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float key_float(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }
__device__ __forceinline__ float warp_min_redux(float v) {
  return key_float(__reduce_min_sync(0xffffffffu, float_key(v)));
}
__device__ __forceinline__ float warp_max_redux(float v) {
  return key_float(__reduce_max_sync(0xffffffffu, float_key(v)));
}

// n / d for 0 <= n < 2^11 and 1 <= d <= 64 by a multiply with ceil(2^20 / d): the error
// n * (ceil(2^20/d) - 2^20/d) / 2^20 < 2^-9 stays below the 1/d gap to the next integer
struct DivTable {
  int m[65];
  constexpr DivTable() : m() {
    for (int d = 1; d <= 64; d++) m[d] = ((1 << 20) + d - 1) / d;
  }
};
__constant__ DivTable c_div = DivTable();
__device__ __forceinline__ int div_small(int n, int d) { return (n * c_div.m[d]) >> 20; }

__device__ __forceinline__ int lowest_bit(unsigned m) { return __ffs(m) - 1; }
__device__ __forceinline__ int lowest_bit(unsigned long long m) { return __ffsll(m) - 1; }

// 4-byte asynchronous global -> shared copy (cp.async, sm_80+), its commit and wait
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

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
  PPItem *items;    // tile-major, heaviest bucket first
  int32_t *sched;   // schedule words, layout in sched_ints()
  int64_t item_cap;
  int t_lo, t_hi;   // tiles of this force launch; its queue head is sched_head(t_lo, t_hi)
  float *vp;
  float mass2, kick, app, app2;
  float cea, ka;  // softening-law constants 2/app and (1/35)/app^2 (0 without softening)
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

// Schedule words (int32), for ntile tiles: [0, 32 ntile) item counts per (tile, bucket), turned
// into the first item slot of each (tile, bucket) by k_pp_offsets; [32 ntile, 64 ntile) cursors;
// then ntile + 1 tile bases (first item of each tile, and the total); then ntile + 1 queue
// heads: a launch over tiles [t_lo, t_hi) uses head t_lo, one over all tiles head ntile, so
// launches over disjoint tile ranges never share a head.
__host__ __device__ inline int64_t sched_base(int ntile) { return 2 * (int64_t)kBuckets * ntile; }
__host__ __device__ inline int64_t sched_head(int ntile, int t_lo, int t_hi) {
  return sched_base(ntile) + ntile + 1 + (t_hi - t_lo == ntile ? ntile : t_lo);
}

// cost bucket of a chunk with ni i-particles and nj candidates, heavy = high index:
// the warp walks the candidates in floor(32/ni) lane groups
__device__ __forceinline__ int cost_bucket(int ni, int64_t nj) {
  int64_t c = nj / (32 / max(ni, 1));
  if (c < 1) c = 1;
  int b = 63 - __clzll(c);
  return b > kBuckets - 1 ? kBuckets - 1 : b;
}

// Enumerate the chunks of the interior PP cells; pass 0 counts items per (tile, bucket),
// pass 1 writes them tile by tile, heaviest bucket first inside a tile.  A cell's full chunks
// share one bucket and its remainder chunk has another, so a thread reserves its slots with at
// most two shared-memory atomics.
template <int PASS, int C>
__global__ void __launch_bounds__(256) k_pp_items(PPK p) {
  __shared__ int sc[kBuckets], sbase[kBuckets];
  const int t = blockIdx.y;
  int32_t *cnt = p.sched + (int64_t)kBuckets * t;                     // counts, then first slots
  int32_t *cur = p.sched + (int64_t)kBuckets * (p.ntile + t);         // cursors
  if (threadIdx.x < kBuckets) sc[threadIdx.x] = 0;
  __syncthreads();
  const TilePP tp = p.tiles[t];
  const int rcp = tp.rcp, S = tp.S, npg = p.nt * rcp;
  const int64_t ncell = (int64_t)npg * npg * npg;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int nfull = 0, bfull = 0, brem = -1, ni = 0, i0 = 0;
  int64_t g = 0;
  PPItem it{};
  if (c < ncell) {
    // cell coordinates in 32-bit arithmetic when the tile's cells fit (64-bit division is a long
    // software sequence)
    int x, y, z;
    if (ncell <= 0xffffffffLL) {
      const unsigned u = (unsigned)c, n = (unsigned)npg, q = u / n, qq = q / n;
      x = (int)(u - q * n) + rcp;
      y = (int)(q - qq * n) + rcp;
      z = (int)qq + rcp;
    } else {
      x = (int)(c % npg) + rcp;
      y = (int)((c / npg) % npg) + rcp;
      z = (int)(c / ((int64_t)npg * npg)) + rcp;
    }
    g = tp.cell0 + ((int64_t)z * S + y) * S + x;
    i0 = p.cs[g];
    ni = p.cs[g + 1] - i0;
    // Sparse neighbouring cells along x share an item when their particles fit one chunk and
    // they lie in one subtile: an aligned group of four cells (at least three occupied), else
    // an aligned pair (both occupied).  The item's stencil rows are `span` cells longer, which
    // walks fewer candidates than separate items and saves their per-item work; the other
    // cells of the group make no item.  Every cell of a group decides the same way.
    int span = 0;
    const int lxi = x - rcp;
    {
      auto count_at = [&](int lx) {
        const int64_t gg = g + (lx - lxi);
        return p.cs[gg + 1] - p.cs[gg];
      };
      // the PP range is set per subtile: a group inside one subtile shares it (groups across a
      // subtile boundary are not formed)
      auto same_range = [&](int lx0, int n) { return lx0 / (rcp * p.ntt) == (lx0 + n - 1) / (rcp * p.ntt); };
      const int h4 = lxi & ~3, h2 = lxi & ~1;
      int tot4 = 0, occ4 = 0;
      if (h4 + 3 < npg)
        for (int k = 0; k < 4; k++) {
          const int cnt = count_at(h4 + k);
          tot4 += cnt;
          occ4 += cnt > 0 ? 1 : 0;
        }
      if (h4 + 3 < npg && tot4 <= C && occ4 >= 3 && same_range(h4, 4)) {
        if (lxi == h4) {
          ni = tot4;
          span = 3;
        } else {
          ni = 0;
        }
      } else if (h2 + 1 < npg) {
        const int n0 = count_at(h2), n1 = count_at(h2 + 1);
        if (n0 > 0 && n1 > 0 && n0 + n1 <= C && same_range(h2, 2)) {
          if (lxi == h2) {
            ni = n0 + n1;
            span = 1;
          } else {
            ni = 0;
          }
        }
      }
    }
    if (ni > 0) {
      const float rc = cell_range(p, t, x, y, z, rcp);
      const int R = stencil_radius(rc, rcp, p.rcs);
      if (R > rcp) atomicOr(p.err, 1 << CUBE_ERR_INVALID);  // beyond the one coarse-cell halo
      const float h = (float)p.rcs / (float)rcp;
      const int Rc = min(R, rcp);
      it.cell = (uint32_t)g;
      it.dims = (rcp << 8) | (Rc << 16) | (span << 24);
      it.rc = rc;
      it.cep = PairLaw::cep_of(rc);
      it.k35 = PairLaw::k35_of(rc);
      it.h = h;
      it.rc2 = rc * rc;
      int64_t nj = 0;
      for (int dz = -Rc; dz <= Rc; dz++)
        for (int dy = -Rc; dy <= Rc; dy++) {
          if (!row_needed(dy, dz, h, rc * rc)) continue;
          const int64_t b = g + ((int64_t)dz * S + dy) * S;
          nj += p.cs[b + Rc + 1 + span] - p.cs[b - Rc];
        }
      nfull = ni / C;
      bfull = cost_bucket(C, nj);
      if (ni % C) brem = cost_bucket(ni % C, nj);
    }
  }
  int rfull = 0, rrem = 0;
  if (nfull) rfull = atomicAdd(&sc[bfull], nfull);
  if (brem >= 0) rrem = atomicAdd(&sc[brem], 1);
  __syncthreads();
  if (threadIdx.x < kBuckets) {
    const int n = sc[threadIdx.x];
    if (PASS == 0) {
      if (n) atomicAdd(&cnt[threadIdx.x], n);
    } else {
      sbase[threadIdx.x] = cnt[threadIdx.x] + (n ? atomicAdd(&cur[threadIdx.x], n) : 0);
    }
  }
  if (PASS == 1) {
    __syncthreads();
    const int64_t f0 = (int64_t)sbase[bfull] + rfull;
    const int dims = it.dims;
    for (int k = 0; k < nfull; k++) {
      it.i0 = i0 + k * C;
      it.dims = dims | C;
      if (f0 + k < p.item_cap) p.items[f0 + k] = it;
      else atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
    }
    if (brem >= 0) {
      const int64_t slot = (int64_t)sbase[brem] + rrem;
      it.i0 = i0 + nfull * C;
      it.dims = dims | (ni - nfull * C);
      if (slot < p.item_cap) p.items[slot] = it;
      else atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
    }
  }
}

// Between the two item passes: turn the (tile, bucket) counts into first slots, tiles in
// order and buckets heaviest first inside a tile, and record the tile bases.  One warp.
__global__ void k_pp_offsets(int32_t *sched, int ntile) {
  const int lane = threadIdx.x;
  int32_t *base = sched + sched_base(ntile);
  int acc = 0;
  for (int t = 0; t < ntile; t++) {
    const int c = sched[kBuckets * t + lane];
    int incl = c;  // inclusive sum over the heavier buckets b' >= lane
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_down_sync(0xffffffffu, incl, o);
      if (lane + o < 32) incl += v;
    }
    if (lane == 0) base[t] = acc;
    sched[kBuckets * t + lane] = acc + incl - c;
    acc += __shfl_sync(0xffffffffu, incl, 0);
  }
  if (lane == 0) base[ntile] = acc;
}

// COUNT = false: forces and kick.  COUNT = true: only count the accepted ordered
// pairs 0 < r^2 < rc^2 (the algorithmic work of the kick, for the roofline).
// Shape: C i-particles per item, J staged candidates per flush, pair loop unrolled U times,
// registers budgeted for B resident blocks per SM, pair law on packed f32x2 arithmetic (PK).
template <bool COUNT, int C, int J, int U, int B, bool PK>
__global__ void __launch_bounds__(kPPThreads, B) k_pp_force(PPK p) {
  // a flush has at most ceil(J / floor(32 / C)) rounds (packed: pair rounds, two candidates
  // each), one bit per round and lane in the soft-pair mask
  constexpr int kNg = 32 / C;
  constexpr int kBits = PK ? (J + 2 * kNg - 1) / (2 * kNg) : (J + kNg - 1) / kNg;
  static_assert(kBits <= 64, "at most 64 soft-pair bits per flush");
  static_assert(!(COUNT && PK), "the pair count runs the scalar loop");
  using Mask = typename std::conditional<(kBits > 32), unsigned long long, unsigned>::type;
  extern __shared__ float4 pp_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  char *wbase = reinterpret_cast<char *>(pp_smem) + warp * pp_smem_warp(J, PK);
  float4 *buf = reinterpret_cast<float4 *>(wbase);  // scalar staging: float4 [J + 32]
  float *X = reinterpret_cast<float *>(wbase);      // packed staging: planes of J + 64 floats
  float *Y = X + (J + 64), *Z = Y + (J + 64);
  // (end of the row in the walk, start - walk offset)
  int2 *rows = reinterpret_cast<int2 *>(wbase + pp_stage_bytes(J, PK));
  float *const ks = reinterpret_cast<float *>(rows + kMaxRows) + lane;  // field f at ks[32 f]
  float *const bbox = reinterpret_cast<float *>(rows + kMaxRows) + 32 * kLaneFields;
  PPItem *const batch = reinterpret_cast<PPItem *>(bbox + 8);
  int *const tcache = reinterpret_cast<int *>(bbox + 6);  // cell and walk of the row table
  if (lane == 0) tcache[0] = -1;
  __syncwarp();
  for (int f = 6; f < 10; f++) ks[32 * f] = 0.f;  // f2, |v| maxima
  unsigned long long npairs = 0;
  // The warp takes kPop consecutive items per queue pop (one atomic and one load for all of
  // them); the items of a bucket cost about the same, and the lightest come last.
  for (int nb = 0, b = 0;; b++) {
    if (b == nb) {
      // items [first, last) of tiles [t_lo, t_hi), popped through this launch's own queue head
      const int32_t *tbase = p.sched + sched_base(p.ntile);
      const int first = tbase[p.t_lo];
      const int last = (int)min((int64_t)tbase[p.t_hi], p.item_cap);
      int it = 0;
      if (lane == 0) it = first + atomicAdd(p.sched + sched_head(p.ntile, p.t_lo, p.t_hi), kPop);
      it = __shfl_sync(0xffffffffu, it, 0);
      if (it >= last) break;
      nb = min(kPop, last - it);
      b = 0;
      __syncwarp();
      if (lane < 2 * nb) reinterpret_cast<int4 *>(batch)[lane] = reinterpret_cast<const int4 *>(p.items + it)[lane];
      __syncwarp();
    }
    const PPItem &item = batch[b];  // read from shared memory where used
    const int64_t g = (int64_t)item.cell;
    const int ni = item.dims & 0xff, R = (item.dims >> 16) & 0xff, span = item.dims >> 24;
    const int S = ((item.dims >> 8) & 0xff) * (p.nt + 2);
    const float rc2 = item.rc2;
    PairLaw law;
    law.init(item);
    // lanes = ngrp groups of ni lanes; group `grp` walks every ngrp-th candidate
    const int ngrp = 32 / ni;
    const int grp = div_small(lane, ni), il = lane - grp * ni;
    const bool has_i = grp < ngrp;  // the 32 mod ni leftover lanes idle
    const float4 pi = p.spos[item.i0 + il];
    bool boxed = false;  // the bounding box is taken once pi has arrived (after the first row table)
    for (int f = 0; f < 6; f++) ks[32 * f] = 0.f;  // Kahan sums of this item
    int nbuf = 0;  // staged candidates (warp-uniform)
    // Evaluate the staged candidates: group grp takes buf[grp + k*ngrp] in round k.  The loop
    // bound is the same for every lane (no divergent loop exits): the slots past nbuf hold a
    // far-away sentinel that the r < rc mask drops, and the lanes of an incomplete last group
    // (grp == ngrp) compute values that the group merge below never reads.  The main loop has
    // no branch: pairs inside the softening length (r <= app, common only in dense clumps) are
    // masked out of it and their rounds recorded in a bit mask (at most 32 rounds per flush);
    // a second loop then evaluates exactly those pairs, one per lane per step.
    // Packed: candidates 2m and 2m + 1 form pair slot m, and group grp takes slots grp + k*ngrp;
    // its two halves are summed separately and added at the end of the flush.
    auto flush_packed = [&]() {
      X[nbuf + lane] = 1e18f;
      Y[nbuf + lane] = 1e18f;
      Z[nbuf + lane] = 1e18f;
      X[nbuf + 32 + lane] = 1e18f;
      Y[nbuf + 32 + lane] = 1e18f;
      Z[nbuf + 32 + lane] = 1e18f;
      __syncwarp();
      float2 px = dup(0.f), py = dup(0.f), pz = dup(0.f);
      const int nround = div_small(nbuf + 2 * ngrp - 1, 2 * ngrp);
      Mask softmask = 0u, bit = 1u;
      const float2 *X2 = reinterpret_cast<const float2 *>(X);
      const float2 nx = dup(-pi.x), ny = dup(-pi.y), nz = dup(-pi.z);
      int m = grp;
#pragma unroll U
      for (int k = 0; k < nround; k++, m += ngrp, bit <<= 1) {
        const float2 dx = add2(X2[m], nx), dy_ = add2(X2[m + (J + 64) / 2], ny),
                     dz_ = add2(X2[m + (J + 64)], nz);
        const float2 r2 = fma2(dx, dx, fma2(dy_, dy_, mul2(dz_, dz_)));
        float2 s = law.scale2(r2);
        const bool fx = r2.x > p.app2, fy = r2.y > p.app2;
        s.x = fx & (r2.x < rc2) ? s.x : 0.0f;
        s.y = fy & (r2.y < rc2) ? s.y : 0.0f;
        if ((!fx & (r2.x > 0.0f)) | (!fy & (r2.y > 0.0f))) softmask |= bit;
        px = fma2(s, dx, px);
        py = fma2(s, dy_, py);
        pz = fma2(s, dz_, pz);
      }
      if (!has_i) softmask = 0u;
      // a flagged pair round holds one or two soft pairs: both halves are tested again
      while (__any_sync(0xffffffffu, softmask != 0u)) {
        if (softmask) {
          const int c = 2 * (grp + lowest_bit(softmask) * ngrp);
          softmask &= softmask - 1u;
#pragma unroll
          for (int e = 0; e < 2; e++) {
            const float dx = X[c + e] - pi.x, dy_ = Y[c + e] - pi.y, dz_ = Z[c + e] - pi.z;
            const float r2 = fmaf(dx, dx, fmaf(dy_, dy_, dz_ * dz_));
            if ((r2 <= p.app2) & (r2 > 0.0f)) {
              const float s = law.soft(r2, p.cea, p.ka);
              px.x = fmaf(s, dx, px.x);
              py.x = fmaf(s, dy_, py.x);
              pz.x = fmaf(s, dz_, pz.x);
            }
          }
        }
      }
      kahan_add(ks[0], ks[32], px.x + px.y);
      kahan_add(ks[64], ks[96], py.x + py.y);
      kahan_add(ks[128], ks[160], pz.x + pz.y);
      nbuf = 0;
      __syncwarp();
    };
    auto flush = [&]() {
      if constexpr (PK) {
        flush_packed();
        return;
      }
      buf[nbuf + lane] = make_float4(1e18f, 1e18f, 1e18f, 0.f);
      __syncwarp();
      float px = 0.f, py = 0.f, pz = 0.f;
      const int nround = div_small(nbuf + ngrp - 1, ngrp);
      Mask softmask = 0u, bit = 1u;
      const float4 *bp = buf + grp;
#pragma unroll U
      for (int k = 0; k < nround; k++, bp += ngrp, bit <<= 1) {
        const float4 pj = *bp;
        const float dx = pj.x - pi.x, dy_ = pj.y - pi.y, dz_ = pj.z - pi.z;
        const float r2 = fmaf(dx, dx, fmaf(dy_, dy_, dz_ * dz_));
        if (COUNT) {
          npairs += (r2 < rc2) & (r2 > 0.0f) & has_i ? 1ull : 0ull;  // r = 0: the particle itself
        } else {
          // evaluated for every candidate and masked: a divergent accept branch would
          // run on nearly every round of a 32-lane warp anyway
          float s = law.scale(r2);
          s = (r2 < rc2) & (r2 > p.app2) ? s : 0.0f;
          softmask |= (r2 <= p.app2) & (r2 > 0.0f) & has_i ? bit : 0u;
          px = fmaf(s, dx, px);
          py = fmaf(s, dy_, py);
          pz = fmaf(s, dz_, pz);
        }
      }
      if (!COUNT) {
        while (__any_sync(0xffffffffu, softmask != 0u)) {
          if (softmask) {
            const int k = lowest_bit(softmask);
            softmask &= softmask - 1u;
            const float4 pj = buf[grp + k * ngrp];
            const float dx = pj.x - pi.x, dy_ = pj.y - pi.y, dz_ = pj.z - pi.z;
            const float s = law.soft(fmaf(dx, dx, fmaf(dy_, dy_, dz_ * dz_)), p.cea, p.ka);
            px = fmaf(s, dx, px);
            py = fmaf(s, dy_, py);
            pz = fmaf(s, dz_, pz);
          }
        }
        kahan_add(ks[0], ks[32], px);
        kahan_add(ks[64], ks[96], py);
        kahan_add(ks[128], ks[160], pz);
      }
      nbuf = 0;
      __syncwarp();
    };
    // The needed stencil rows are laid end to end in a table of up to kMaxRows rows: row k
    // covers walk positions [rows[k-1].x, rows[k].x), and walk position v is particle
    // v + rows[k].y.  Stencils with more rows (large R) are walked in several tables.
    // Consecutive items of one cell share their stencil: a table that holds the whole stencil is
    // kept for the next item (tcache: its cell, or -1, and its walk length).
    const int side = 2 * R + 1, nr = side * side;
    for (int r0 = 0; r0 < nr;) {
      int nrows = 0, walk = 0;
      const bool reuse = r0 == 0 && tcache[0] == (int)item.cell;
      if (reuse) {
        walk = tcache[1];
        r0 = nr;
      }
      const int rstart = r0;
      for (; r0 < nr && nrows <= kMaxRows - 32; r0 += 32) {
        const int ri = r0 + lane;
        int js = 0, len = 0;
        bool need = false;
        if (ri < nr) {
          const int q = div_small(ri, side);
          const int dz = q - R, dy = ri - q * side - R;
          need = row_needed(dy, dz, item.h, rc2);
          if (need) {
            const int64_t b = g + ((int64_t)dz * S + dy) * S;
            js = p.cs[b - R];
            len = p.cs[b + R + 1 + span] - js;
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, need);
        int incl = len;  // inclusive scan of the lengths (0 for rows not needed)
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        if (need) rows[nrows + __popc(m & ((1u << lane) - 1u))] = make_int2(walk + incl, js - (walk + incl - len));
        nrows += __popc(m);
        walk += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (!reuse && lane == 0) {
        tcache[0] = rstart == 0 && r0 >= nr ? (int)item.cell : -1;
        tcache[1] = walk;
      }
      __syncwarp();
      if (!boxed) {
        // bounding box of the item's particles: candidates farther than rc from it are dropped
        // while staging, so the pair loop below only sees possibly-interacting candidates
        boxed = true;
        const float blx = warp_min_redux(pi.x), bhx = warp_max_redux(pi.x), bly = warp_min_redux(pi.y),
                    bhy = warp_max_redux(pi.y), blz = warp_min_redux(pi.z), bhz = warp_max_redux(pi.z);
        if (lane == 0) {
          *reinterpret_cast<float4 *>(bbox) = make_float4(blx, bly, blz, bhx);
          *reinterpret_cast<float2 *>(bbox + 4) = make_float2(bhy, bhz);
        }
        // the owned particle's velocity is copied in while the item runs
        if (!COUNT && grp == 0 && has_i) {
          const float *v = p.vp + 3 * (int64_t)__float_as_int(pi.w);
          cp_async4(ks + 320, v);
          cp_async4(ks + 352, v + 1);
          cp_async4(ks + 384, v + 2);
        }
        cp_async_commit();
        __syncwarp();
      }
      if (walk == 0) continue;
      // Walk position -> particle.  Each lane's row index only moves forward and stops at the
      // last row (rows[nrows-1].x = walk > v), and the lanes past the end load the last
      // candidate again and drop it, so the loop below has no divergent branch or load.
      int kr = 0;
      auto locate = [&](int v) {
        v = min(v, walk - 1);
        while (__any_sync(0xffffffffu, v >= rows[kr].x)) kr += v >= rows[kr].x ? 1 : 0;
        return v + rows[kr].y;
      };
      float4 nxt = p.spos[locate(lane)];
      for (int vb = 0; vb < walk; vb += 32) {
        const float4 pj = nxt;
        nxt = p.spos[locate(vb + 32 + lane)];  // one step ahead
        const float4 bl = *reinterpret_cast<const float4 *>(bbox);  // (lo x, y, z, hi x)
        const float2 bh = *reinterpret_cast<const float2 *>(bbox + 4);  // (hi y, z)
        const float ex = fmaxf(fmaxf(bl.x - pj.x, pj.x - bl.w), 0.f);
        const float ey = fmaxf(fmaxf(bl.y - pj.y, pj.y - bh.x), 0.f);
        const float ez = fmaxf(fmaxf(bl.z - pj.z, pj.z - bh.y), 0.f);
        const bool keep = (vb + lane < walk) & (ex * ex + ey * ey + ez * ez < rc2);
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          const int q = nbuf + __popc(m & ((1u << lane) - 1u));
          if constexpr (PK) {
            X[q] = pj.x;
            Y[q] = pj.y;
            Z[q] = pj.z;
          } else {
            buf[q] = pj;
          }
        }
        nbuf += __popc(m);
        if (nbuf > J - 32) flush();
      }
      __syncwarp();  // the next table overwrites this one
    }
    if (nbuf) flush();
    // merge the lane groups of each i-particle (tree over groups, stride s*ni lanes);
    // Kahan c is the negated low part
    float hx = ks[0], lx = -ks[32], hy = ks[64], ly = -ks[96], hz = ks[128], lz = -ks[160];
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
      ks[192] = fmaxf(ks[192], ax * ax + ay * ay + az * az);
      const int64_t ip = (int64_t)__float_as_int(pi.w);
      float *v = p.vp + 3 * ip;
      cp_async_wait_all();
      const float v0 = ks[320] + ax * p.kick, v1 = ks[352] + ay * p.kick, v2 = ks[384] + az * p.kick;
      v[0] = v0;
      v[1] = v1;
      v[2] = v2;
      ks[224] = fmaxf(ks[224], fabsf(v0));
      ks[256] = fmaxf(ks[256], fabsf(v1));
      ks[288] = fmaxf(ks[288], fabsf(v2));
    }
  }
  if (COUNT) {
    for (int o = 16; o; o >>= 1) npairs += __shfl_xor_sync(0xffffffffu, npairs, o);
    if (lane == 0) atomicAdd(p.pairs, npairs);
    return;
  }
  const float f2w = warp_max(ks[192]);
  if (lane == 0) atomic_max_nonneg(&p.out[1], f2w);
  if (p.want_vmax) {
    const float vm0 = warp_max(ks[224]), vm1 = warp_max(ks[256]), vm2 = warp_max(ks[288]);
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
  p.sched = a.sched;
  p.item_cap = a.item_cap;
  p.t_lo = 0;
  p.t_hi = L.ntile;
  p.vp = a.vp;
  p.mass2 = a.mass2;
  p.kick = a.kick;
  p.app = L.app;
  p.app2 = L.app * L.app;
  p.cea = L.app > 0.f ? 2.0f / L.app : 0.f;
  p.ka = L.app > 0.f ? (1.0f / 35.0f) / (L.app * L.app) : 0.f;
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

size_t sched_ints(int ntile) { return (size_t)sched_base(ntile) + 2 * ((size_t)ntile + 1); }
int64_t sched_total_index(int ntile) { return sched_base(ntile) + ntile; }

int pp_num_shapes() { return kNumShapes; }
PPShapeDesc pp_shape_desc(int i) { return kShapes[i >= 0 && i < kNumShapes ? i : 0]; }
int pp_min_chunk() { return kMinChunk; }

template <int C>
static void launch_items_c(const PPK &p, dim3 grid, cudaStream_t s, int32_t *sched, int ntile) {
  k_pp_items<0, C><<<grid, 256, 0, s>>>(p);
  k_pp_offsets<<<1, 32, 0, s>>>(sched, ntile);
  k_pp_items<1, C><<<grid, 256, 0, s>>>(p);
}

void launch_pp_items(const PPArgs &a, cudaStream_t s) {
  PPK p = make_ppk(a);
  cudaMemsetAsync(a.sched, 0, sizeof(int32_t) * sched_ints(a.L->ntile), s);
  dim3 grid((unsigned)((p.max_cells + 255) / 256), (unsigned)a.L->ntile);
  switch (pp_shape_desc(a.pairs ? 0 : a.shape).chunk) {
    case 4: launch_items_c<4>(p, grid, s, a.sched, a.L->ntile); break;
    case 16: launch_items_c<16>(p, grid, s, a.sched, a.L->ntile); break;
    case 32: launch_items_c<32>(p, grid, s, a.sched, a.L->ntile); break;
    default: launch_items_c<8>(p, grid, s, a.sched, a.L->ntile); break;
  }
}

// One persistent block per resident slot: blocks beyond the resident count would only start
// once the queue is empty.  The shared-memory attribute is set and the count looked up once per
// kernel (slot = shape, or the pair-count kernel) and device: the attribute is per device.
constexpr int kMaxDevices = 64;
template <bool COUNT, int S>
static void launch_force_shape(const PPK &p, int num_sms, cudaStream_t s) {
  constexpr PPShapeDesc d = COUNT ? kCountShape : kShapes[S];
  constexpr size_t smem = pp_smem_block(d.jtile, d.packed != 0);
  auto fn = k_pp_force<COUNT, d.chunk, d.jtile, d.unroll, d.blocks, d.packed != 0>;
  static int per_sm[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int n = 0;
  if (dev < 0 || dev >= kMaxDevices || !per_sm[dev]) {
    cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void *)fn, kPPThreads, smem);
    n = n > 0 ? n : 1;
    if (dev >= 0 && dev < kMaxDevices) per_sm[dev] = n;
  } else {
    n = per_sm[dev];
  }
  fn<<<n * num_sms, kPPThreads, smem, s>>>(p);
}

template <int... I>
static void launch_force_any(int shape, const PPK &p, int num_sms, cudaStream_t s, std::integer_sequence<int, I...>) {
  ((shape == I ? launch_force_shape<false, I>(p, num_sms, s) : void()), ...);
}

void launch_pp_force(const PPArgs &a, cudaStream_t s, int t_lo, int t_hi) {
  PPK p = make_ppk(a);
  if (t_hi < 0) t_hi = a.L->ntile;
  p.t_lo = t_lo;
  p.t_hi = t_hi;
  if (a.pairs) {
    launch_force_shape<true, 0>(p, a.num_sms, s);  // kCountShape: the work list of shape 0
  } else {
    const int shape = a.shape >= 0 && a.shape < kNumShapes ? a.shape : 0;
    launch_force_any(shape, p, a.num_sms, s, std::make_integer_sequence<int, kNumShapes>{});
  }
}

}  // namespace cube
