// PM3 fine-mesh force (kick.f90:403-568, pm3_fft_cuda.cu:276-391).
//
// Pipeline per batch of meshes:
//   deposit  TSC weights of every particle of the job's coarse cells into the
//            mesh (kick.f90:420-468); one warp per coarse cell, float atomics
//            (the cost follows the particles, not the mesh, which matters for
//            clustered boxes where most mesh bricks are nearly empty);
//   R2C      cuFFT;
//   k-space  the potential spectrum: rho(k) * G(k) * mass / n^3, in place
//            (kick.f90:472-491 and the 1/nwork^3 of kick.f90:552);
//   C2R      cuFFT, one transform per mesh;
//   force    the 4-point difference of potential_to_force (kick.f90:545-568)
//            on the periodic FFT mesh, four x points per thread, writing the
//            three force arrays and the max |F|^2 over the physical mesh
//            points (kick.f90:494) in the same pass;
//   gather   TSC gather of the force at each active particle and the kick
//            vp += dv * a_mid*dt/(6 pi) (kick.f90:497-540).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace cube {

struct PM3K {
  int n, nt, nte, ncb;
  int64_t n3, nk;  // mesh points, half-spectrum points per slot
  int rdep[3], ract[3];
  int wrap, shift;
  double scale;
  const MeshJob *jobs;
  int njobs;
  const int16_t *xp;
  const int32_t *rhoc;
  const int64_t *cell_base;
  float *rho;           // density, then potential [slot][n^3]
  cufftComplex *rhok;
  float *force;  // [slot][3][n^3]
  const float *green;
  float gscale;  // mass / n^3
  float kick;
  float *vp;
  float *out;
  int want_vmax;
  int fphys_lo, fphys_n;
  int nslots;
  int32_t *err;
  int32_t *brick_ctr;
};

// a + d into [0, n) for |d| < n
__device__ __forceinline__ int64_t wrap_near(int64_t a, int64_t n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

// TSC weights in real(4) from a real(8) coordinate (kick.f90:439-445)
__device__ __forceinline__ int64_t tsc(double m, float w[3]) {
  const double f = floor(m);
  const float l3 = (float)(m - f);
  w[0] = __fmul_rn(1.0f - l3, 1.0f - l3) * 0.5f;
  w[2] = __fmul_rn(l3, l3) * 0.5f;
  w[1] = 1.0f - w[0] - w[2];
  return (int64_t)f;
}

__global__ void __launch_bounds__(kWarps * 32) k_deposit(PM3K p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t cells = (int64_t)p.rdep[0] * p.rdep[1] * p.rdep[2];
  const int64_t wid = (int64_t)blockIdx.x * kWarps + warp;
  if (wid >= cells * p.njobs) return;
  const int j = (int)(wid / cells);
  const int64_t r = wid - (int64_t)j * cells;
  const MeshJob J = p.jobs[j];
  const int ci = J.lo[0] + (int)(r % p.rdep[0]);
  const int cj = J.lo[1] + (int)((r / p.rdep[0]) % p.rdep[1]);
  const int ck = J.lo[2] + (int)(r / ((int64_t)p.rdep[0] * p.rdep[1]));
  const int64_t cidx = (((int64_t)J.t * p.nte + ck) * p.nte + cj) * p.nte + ci;
  const int np = p.rhoc[cidx];
  const int64_t base = p.cell_base[cidx];
  float *R = p.rho + (int64_t)J.slot * p.n3;
  const int64_t n = p.n;
  for (int l = lane; l < np; l += 32) {
    const int16_t *q = p.xp + 3 * (base + l);
    float wx[3], wy[3], wz[3];
    const int64_t ix = tsc(decode_pos(ci - p.ncb, q[0]) * p.scale - J.off[0], wx) + p.shift;
    const int64_t iy = tsc(decode_pos(cj - p.ncb, q[1]) * p.scale - J.off[1], wy) + p.shift;
    const int64_t iz = tsc(decode_pos(ck - p.ncb, q[2]) * p.scale - J.off[2], wz) + p.shift;
    // the three x points of a row are one vector reduction when they lie in a 16-byte
    // window, else a pair and a single (rows are 16-byte aligned when n % 4 == 0)
    const bool vec = (n % 4 == 0) && ix >= 1 && ix + 1 < n;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int64_t Z = iz + c - 1;
      if (p.wrap) Z = wrap_near(Z, n); else if (Z < 0 || Z >= n) continue;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        int64_t Y = iy + b - 1;
        if (p.wrap) Y = wrap_near(Y, n); else if (Y < 0 || Y >= n) continue;
        float *row = R + (Z * n + Y) * n;
        const float w0 = (wx[0] * wy[b]) * wz[c], w1 = (wx[1] * wy[b]) * wz[c], w2 = (wx[2] * wy[b]) * wz[c];
        if (vec) {
          const int64_t x0 = ix - 1, o = x0 & 3, b4 = x0 - o;
          if (o == 0) {
            atomicAdd(reinterpret_cast<float4 *>(row + b4), make_float4(w0, w1, w2, 0.f));
          } else if (o == 1) {
            atomicAdd(reinterpret_cast<float4 *>(row + b4), make_float4(0.f, w0, w1, w2));
          } else if (o == 2) {
            atomicAdd(reinterpret_cast<float2 *>(row + b4 + 2), make_float2(w0, w1));
            atomicAdd(row + b4 + 4, w2);
          } else {
            atomicAdd(row + b4 + 3, w0);
            atomicAdd(reinterpret_cast<float2 *>(row + b4 + 4), make_float2(w1, w2));
          }
          continue;
        }
        const float wr[3] = {w0, w1, w2};
#pragma unroll
        for (int a = 0; a < 3; a++) {
          int64_t X = ix + a - 1;
          if (p.wrap) X = wrap_near(X, n); else if (X < 0 || X >= n) continue;
          atomicAdd(row + X, wr[a]);
        }
      }
    }
  }
}

// potential spectrum in place: rhok[slot] *= G(k) * mass / n^3
__global__ void k_kspace(PM3K p) {
  const int64_t total = p.nk * p.nslots;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e % p.nk;
    const float g = p.green[k] * p.gscale;
    const cufftComplex c = p.rhok[e];
    p.rhok[e] = make_float2(c.x * g, c.y * g);
  }
}

// weights of potential_to_force at offsets -2, -1, +1, +2 (parameters.f90:49-50, a = real(4) 4/3)
struct FDW {
  float m2, m1, p1, p2;
  __device__ __forceinline__ FDW() {
    const float a = 4.0f / 3.0f;
    m2 = (a - 1.0f) / 4.0f;
    m1 = -a / 2.0f;
    p1 = a / 2.0f;
    p2 = (1.0f - a) / 4.0f;
  }
  __device__ __forceinline__ float operator()(float fm2, float fm1, float fp1, float fp2) const {
    return fm2 * m2 + fm1 * m1 + fp1 * p1 + fp2 * p2;  // sum(phi(i_n) * weight), kick.f90:562-564
  }
};

__device__ __forceinline__ bool in_phys(const PM3K &p, int64_t x, int64_t y, int64_t z) {
  return x >= p.fphys_lo && x < p.fphys_lo + p.fphys_n && y >= p.fphys_lo && y < p.fphys_lo + p.fphys_n &&
         z >= p.fphys_lo && z < p.fphys_lo + p.fphys_n;
}

// Force from the potential on the periodic mesh (n % 4 == 0).  A block owns 32 float4 columns
// (128 x points) of kFzRows rows and marches through kFzChunk planes: each thread keeps the
// five planes z-2 .. z+2 of its own column in registers and loads one new float4 per plane;
// x neighbours come from the adjacent lanes (the edge lanes load theirs), y neighbours from a
// shared tile of the block's rows plus two halo rows on each side.  Each potential value is
// thus read about once from DRAM.  Stores go to the three force arrays (an interleaved
// (fx, fy, fz, 0) layout measured twice as slow in the gather); |F|^2 of the physical points is
// reduced into out[0].
constexpr int kFzRows = 8;
constexpr int kFzChunk = 32;

__device__ __forceinline__ float4 shfl_f4(float4 v, int delta, bool up) {
  float4 r;
  r.x = up ? __shfl_up_sync(0xffffffffu, v.x, delta) : __shfl_down_sync(0xffffffffu, v.x, delta);
  r.y = up ? __shfl_up_sync(0xffffffffu, v.y, delta) : __shfl_down_sync(0xffffffffu, v.y, delta);
  r.z = up ? __shfl_up_sync(0xffffffffu, v.z, delta) : __shfl_down_sync(0xffffffffu, v.z, delta);
  r.w = up ? __shfl_up_sync(0xffffffffu, v.w, delta) : __shfl_down_sync(0xffffffffu, v.w, delta);
  return r;
}

__global__ void __launch_bounds__(kFzRows * 32) k_force_zm(PM3K p) {
  __shared__ float4 tile[kFzRows + 4][32];
  const FDW w;
  const int lane = threadIdx.x & 31, wy = threadIdx.x >> 5;
  const int64_t n = p.n, n4 = p.n / 4;
  const int nzc = (p.n + kFzChunk - 1) / kFzChunk;
  const int64_t slot = blockIdx.z / nzc;
  const int64_t z0 = (int64_t)(blockIdx.z % nzc) * kFzChunk, z1 = min(z0 + kFzChunk, n);
  const int64_t x4 = (int64_t)blockIdx.x * 32 + lane, y0 = (int64_t)blockIdx.y * kFzRows, y = y0 + wy;
  const bool act = x4 < n4 && y < n;
  // idle lanes read a valid column; rows past n march the periodic image row, which the
  // rows below them read as their y neighbours
  const int64_t xs = min(x4, n4 - 1), ys = wrap_near(y, n);
  const float4 *phi = reinterpret_cast<const float4 *>(p.rho + slot * p.n3);
  auto at = [&](int64_t xx4, int64_t yy, int64_t zz) {
    return __ldg(phi + (wrap_near(zz, n) * n + wrap_near(yy, n)) * n4 + wrap_near(xx4, n4));
  };
  float4 cm2 = at(xs, ys, z0 - 2), cm1 = at(xs, ys, z0 - 1), c0 = at(xs, ys, z0), cp1 = at(xs, ys, z0 + 1);
  float4 *F = reinterpret_cast<float4 *>(p.force + slot * 3 * p.n3) + ys * n4 + xs;
  const int64_t plane4 = n * n4;
  float m = 0.f;
  for (int64_t z = z0; z < z1; z++) {
    const float4 cp2 = at(xs, ys, z + 2);
    tile[wy + 2][lane] = c0;
    if (wy < 4) {  // halo rows y0-2, y0-1 (warps 0, 1) and y0+kFzRows, y0+kFzRows+1 (warps 2, 3)
      const int64_t hy = wy < 2 ? y0 - 2 + wy : y0 + kFzRows + wy - 2;
      tile[wy < 2 ? wy : kFzRows + wy][lane] = at(xs, hy, z);
    }
    float4 l = shfl_f4(c0, 1, true), r = shfl_f4(c0, 1, false);
    if (lane == 0) l = at(xs - 1, ys, z);
    if (lane == 31 || x4 + 1 >= n4) r = at(xs + 1, ys, z);
    __syncthreads();
    const float4 ym2 = tile[wy][lane], ym1 = tile[wy + 1][lane], yp1 = tile[wy + 3][lane],
                 yp2 = tile[wy + 4][lane];
    const float4 fx = make_float4(w(l.z, l.w, c0.y, c0.z), w(l.w, c0.x, c0.z, c0.w), w(c0.x, c0.y, c0.w, r.x),
                                  w(c0.y, c0.z, r.x, r.y));
    const float4 fy = make_float4(w(ym2.x, ym1.x, yp1.x, yp2.x), w(ym2.y, ym1.y, yp1.y, yp2.y),
                                  w(ym2.z, ym1.z, yp1.z, yp2.z), w(ym2.w, ym1.w, yp1.w, yp2.w));
    const float4 fz = make_float4(w(cm2.x, cm1.x, cp1.x, cp2.x), w(cm2.y, cm1.y, cp1.y, cp2.y),
                                  w(cm2.z, cm1.z, cp1.z, cp2.z), w(cm2.w, cm1.w, cp1.w, cp2.w));
    if (act) {
      float4 *Fz = F + z * plane4;
      Fz[0] = fx;
      Fz[n * plane4] = fy;
      Fz[2 * n * plane4] = fz;
      const int64_t x = 4 * x4;
      if (in_phys(p, x, y, z)) m = fmaxf(m, fx.x * fx.x + fy.x * fy.x + fz.x * fz.x);
      if (in_phys(p, x + 1, y, z)) m = fmaxf(m, fx.y * fx.y + fy.y * fy.y + fz.y * fz.y);
      if (in_phys(p, x + 2, y, z)) m = fmaxf(m, fx.z * fx.z + fy.z * fy.z + fz.z * fz.z);
      if (in_phys(p, x + 3, y, z)) m = fmaxf(m, fx.w * fx.w + fy.w * fy.w + fz.w * fz.w);
    }
    __syncthreads();  // the next plane overwrites the tile
    cm2 = cm1;
    cm1 = c0;
    c0 = cp1;
    cp1 = cp2;
  }
  // one update of f2max per block
  __shared__ float mb[kFzRows];
  m = warp_max(m);
  if (lane == 0) mb[wy] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kFzRows; w++) m = fmaxf(m, mb[w]);
    atomic_max_nonneg(&p.out[0], m);
  }
}

// the same, one point per thread, for any n
__global__ void k_force(PM3K p) {
  const FDW w;
  const int64_t n = p.n;
  const int64_t total = p.n3 * p.nslots;
  float m = 0.f;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t slot = e / p.n3, r = e - slot * p.n3;
    const int64_t x = r % n, y = (r / n) % n, z = r / (n * n);
    const float *phi = p.rho + slot * p.n3;
    auto at = [&](int64_t xx, int64_t yy, int64_t zz) {
      return __ldg(phi + (wrap_near(zz, n) * n + wrap_near(yy, n)) * n + wrap_near(xx, n));
    };
    const float fx = w(at(x - 2, y, z), at(x - 1, y, z), at(x + 1, y, z), at(x + 2, y, z));
    const float fy = w(at(x, y - 2, z), at(x, y - 1, z), at(x, y + 1, z), at(x, y + 2, z));
    const float fz = w(at(x, y, z - 2), at(x, y, z - 1), at(x, y, z + 1), at(x, y, z + 2));
    float *F = p.force + slot * 3 * p.n3 + r;
    F[0] = fx;
    F[p.n3] = fy;
    F[2 * p.n3] = fz;
    if (in_phys(p, x, y, z)) m = fmaxf(m, fx * fx + fy * fy + fz * fz);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&p.out[0], m);
}

__global__ void __launch_bounds__(kWarps * 32, 4) k_gather(PM3K p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t cells = (int64_t)p.ract[0] * p.ract[1] * p.ract[2];
  const int64_t wid = (int64_t)blockIdx.x * kWarps + warp;
  float vm0 = 0.f, vm1 = 0.f, vm2 = 0.f;
  if (wid < cells * p.njobs) {
    const int j = (int)(wid / cells);
    const int64_t r = wid - (int64_t)j * cells;
    const MeshJob J = p.jobs[j];
    const int ci = J.alo[0] + (int)(r % p.ract[0]);
    const int cj = J.alo[1] + (int)((r / p.ract[0]) % p.ract[1]);
    const int ck = J.alo[2] + (int)(r / ((int64_t)p.ract[0] * p.ract[1]));
    const int64_t cidx = (((int64_t)J.t * p.nte + ck) * p.nte + cj) * p.nte + ci;
    const int np = p.rhoc[cidx];
    const int64_t base = p.cell_base[cidx];
    const float *F = p.force + (int64_t)J.slot * 3 * p.n3;
    const int64_t n = p.n, n3 = p.n3;
    for (int l = lane; l < np; l += 32) {
      const int64_t ip = base + l;
      const int16_t *q = p.xp + 3 * ip;
      float wx[3], wy[3], wz[3];
      const int64_t ix = tsc(decode_pos(ci - p.ncb, q[0]) * p.scale - J.off[0], wx) + p.shift;
      const int64_t iy = tsc(decode_pos(cj - p.ncb, q[1]) * p.scale - J.off[1], wy) + p.shift;
      const int64_t iz = tsc(decode_pos(ck - p.ncb, q[2]) * p.scale - J.off[2], wz) + p.shift;
      float d0 = 0.f, d1 = 0.f, d2 = 0.f;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const int64_t Z = p.wrap ? wrap_near(iz + c - 1, n) : iz + c - 1;
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const int64_t Y = p.wrap ? wrap_near(iy + b - 1, n) : iy + b - 1;
#pragma unroll
          for (int a = 0; a < 3; a++) {
            const int64_t X = p.wrap ? wrap_near(ix + a - 1, n) : ix + a - 1;
            const int64_t m = (Z * n + Y) * n + X;
            const float w = (wx[a] * wy[b]) * wz[c];
            d0 += F[m] * w;
            d1 += F[n3 + m] * w;
            d2 += F[2 * n3 + m] * w;
          }
        }
      }
      float *v = p.vp + 3 * ip;
      const float v0 = v[0] + d0 * p.kick, v1 = v[1] + d1 * p.kick, v2 = v[2] + d2 * p.kick;
      v[0] = v0;
      v[1] = v1;
      v[2] = v2;
      vm0 = fmaxf(vm0, fabsf(v0));
      vm1 = fmaxf(vm1, fabsf(v1));
      vm2 = fmaxf(vm2, fabsf(v2));
    }
  }
  if (p.want_vmax) {
    // one update of each maximum per block: a warp per coarse cell would put hundreds of
    // thousands of atomics on the same three words
    __shared__ float vmb[3][kWarps];
    vm0 = warp_max(vm0);
    vm1 = warp_max(vm1);
    vm2 = warp_max(vm2);
    if (lane == 0) {
      vmb[0][warp] = vm0;
      vmb[1][warp] = vm1;
      vmb[2][warp] = vm2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      float m = 0.f;
      for (int w = 0; w < kWarps; w++) m = fmaxf(m, vmb[threadIdx.x][w]);
      atomic_max_nonneg(&p.out[2 + threadIdx.x], m);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Brick kernels for the periodic meshes (wrap = 1): a brick is kBrick^3 mesh points, i.e.
// (kBrick / mc)^3 coarse cells of one job, mc = mesh points per coarse cell.  The bricks of a job
// tile its active cells, and those of all jobs tile the mesh once.  A brick's particles lie in
// (kBrick / mc)^2 rows of (kBrick / mc) coarse cells, and every row is one contiguous run of
// storage, so a block walks them as one flat list.
constexpr int kBrick = 16;               // owned mesh points per brick side
constexpr int kMaxCb = 4;                // coarse cells per brick side (mc >= 4)
constexpr int kMaxRowsPerBrick = kMaxCb * kMaxCb;

struct BrickRows {
  int nrows, total;
  int cb;  // coarse cells per brick side
};

// The brick's rows of coarse cells: first particle, count and the coarse cells' first particles
// (relative to the row), in shared memory.  Contains two block barriers.
__device__ __forceinline__ void brick_rows(const PM3K &p, const MeshJob &J, int cb, int ci0, int cj0, int ck0,
                                          int64_t *rbase, int *rstart, int *rcell, BrickRows &br) {
  const int nrows = cb * cb;
  for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
    const int cj = cj0 + r % cb, ck = ck0 + r / cb;
    const int64_t c0 = (((int64_t)J.t * p.nte + ck) * p.nte + cj) * p.nte + ci0;
    int acc = 0;
    for (int i = 0; i < cb; i++) {
      rcell[r * (kMaxCb + 1) + i] = acc;
      acc += p.rhoc[c0 + i];
    }
    rcell[r * (kMaxCb + 1) + cb] = acc;
    rbase[r] = p.cell_base[c0];
    rstart[r] = acc;  // count for now
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int r = 0; r < nrows; r++) {
      const int c = rstart[r];
      rstart[r] = acc;
      acc += c;
    }
    rstart[nrows] = acc;
  }
  __syncthreads();
  br.nrows = nrows;
  br.total = rstart[nrows];
  br.cb = cb;
}

// Flat particle index k of the brick -> (storage index, coarse cell offsets within the brick).
__device__ __forceinline__ int64_t brick_particle(int k, const BrickRows &br, const int64_t *rbase, const int *rstart,
                                                  const int *rcell, int &di, int &dj, int &dk) {
  int lo = 0, hi = br.nrows - 1;  // last row with rstart <= k
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (rstart[mid] <= k) lo = mid; else hi = mid - 1;
  }
  const int l = k - rstart[lo];
  int i = 0;
  while (i + 1 < br.cb && rcell[lo * (kMaxCb + 1) + i + 1] <= l) i++;
  di = i;
  // cb is 1, 2 or 4 (a brick side of 16 mesh points, at least 4 mesh points per coarse cell)
  dj = lo & (br.cb - 1);
  dk = lo >> (br.cb >> 1);
  return rbase[lo] + l;
}

// brick b of the launch -> job, first coarse cell, first owned mesh point (exact: the offsets of
// periodic jobs are whole mesh points, and the owned points start on a multiple of kBrick)
struct BrickPos {
  int j, ci0, cj0, ck0;
  int64_t X0, Y0, Z0;
};
__device__ __forceinline__ BrickPos brick_pos(const PM3K &p, int64_t b, int cb, const int *ext, const int *lo_of) {
  const int nbx = ext[0] / cb, nby = ext[1] / cb, nbz = ext[2] / cb;
  const int64_t per_job = (int64_t)nbx * nby * nbz;
  BrickPos q;
  q.j = (int)(b / per_job);
  const int64_t r = b - (int64_t)q.j * per_job;
  const MeshJob &J = p.jobs[q.j];
  const int lo[3] = {lo_of == nullptr ? J.alo[0] : J.lo[0], lo_of == nullptr ? J.alo[1] : J.lo[1],
                     lo_of == nullptr ? J.alo[2] : J.lo[2]};
  q.ci0 = lo[0] + (int)(r % nbx) * cb;
  q.cj0 = lo[1] + (int)((r / nbx) % nby) * cb;
  q.ck0 = lo[2] + (int)(r / ((int64_t)nbx * nby)) * cb;
  const int64_t n = p.n;
  q.X0 = wrapi(llrint((double)(q.ci0 - p.ncb) * p.scale - J.off[0]) + p.shift, n);
  q.Y0 = wrapi(llrint((double)(q.cj0 - p.ncb) * p.scale - J.off[1]) + p.shift, n);
  q.Z0 = wrapi(llrint((double)(q.ck0 - p.ncb) * p.scale - J.off[2]) + p.shift, n);
  return q;
}

// ---- mbarrier and bulk-copy helpers (sm_90+) ----
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// arrive on the mbarrier and expect `bytes` of asynchronous copies in the same phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ unsigned long long ns_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr unsigned long long kBulkWaitNs = 1000000000ull;  // bound of one wait for a brick's copies: 1 s
// wait for a phase of the mbarrier, at most kBulkWaitNs; false when the wait gave up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  const unsigned long long t0 = ns_now();
  while (!mbar_try_wait(bar, parity))
    if (ns_now() - t0 > kBulkWaitNs) return false;
  return true;
}
// bulk asynchronous copy global -> this CTA's shared memory, completing on the mbarrier
// (both addresses 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Force and gather in one pass, persistent and warp-specialised: one 1024-thread block per SM
// claims bricks from a work counter.  Its producer warps (the first kFgProd threads) compute a
// brick's force window while its consumer warps gather the previous brick, so the two phases
// overlap instead of alternating behind block barriers.
//   producers: the brick's potential window (the brick plus three points on every side; along
//     x widened to whole 16-byte groups) arrives by one 4-d tensor copy of the ghost-padded
//     potential (cp.async.bulk.tensor, the ghost points hold the periodic images so the box
//     never wraps); the 4-point difference of potential_to_force (kick.f90:545-568) gives the
//     three force components on the brick plus one point on every side, in one of two force
//     buffers, and max |F|^2 of the owned points (kick.f90:494); the brick's row table goes
//     beside it; then the next brick's window is requested.
//   consumers: every active particle of the brick gathers its 27 TSC points from the force
//     buffer and is kicked (kick.f90:497-540).
// The buffers change hands through mbarriers (full: producers -> consumers, empty: back), every
// wait bounded; a decision to stop is voted group-wide, so a group's barriers stay matched.
// The arithmetic (weights, products, summation order) is the one of k_force_zm followed by
// k_gather, and the force arrays never reach HBM.
constexpr int kFgThreads = 1024;
#ifndef CUBE_FG_PRODUCERS
#define CUBE_FG_PRODUCERS 512
#endif
constexpr int kFgProd = CUBE_FG_PRODUCERS;    // producer threads (the first warps of the block)
constexpr int kFgCons = kFgThreads - kFgProd;  // consumer threads
static_assert(kFgProd % 32 == 0 && kFgProd >= 128 && kFgCons >= 128, "whole warps in both groups");
constexpr int kPotX = kBrick + 8, kPotW = kBrick + 6;  // potential window: x 24, y and z 22
constexpr int kForW = kBrick + 2;                      // force window 18^3
constexpr int kPotElems = kPotW * kPotW * kPotX;
constexpr uint32_t kPotBytes = sizeof(float) * kPotElems;
constexpr int kFor3 = kForW * kForW * kForW;
constexpr size_t kFgSmem = (size_t)kPotBytes + 2 * sizeof(float) * 3 * (size_t)kFor3 + 128;  // + alignment slack

struct BrickMeta {
  BrickPos pos;
  int total;  // particles of the brick; -1: no brick (the consumers stop)
  int64_t rbase[kMaxRowsPerBrick];
  int rstart[kMaxRowsPerBrick + 1];
  int rcell[kMaxRowsPerBrick * (kMaxCb + 1)];
};

// row r of brick (pos) into meta: first particle and the coarse cells' offsets (thread r)
__device__ __forceinline__ void meta_row(const PM3K &p, int cb, BrickMeta &mt, int r) {
  const BrickPos &q = mt.pos;
  const int cj = q.cj0 + r % cb, ck = q.ck0 + r / cb;
  const int64_t c0 = (((int64_t)p.jobs[q.j].t * p.nte + ck) * p.nte + cj) * p.nte + q.ci0;
  int acc = 0;
  for (int i = 0; i < cb; i++) {
    mt.rcell[r * (kMaxCb + 1) + i] = acc;
    acc += p.rhoc[c0 + i];
  }
  mt.rcell[r * (kMaxCb + 1) + cb] = acc;
  mt.rbase[r] = p.cell_base[c0];
  mt.rstart[r] = acc;  // count until meta_scan
}
__device__ __forceinline__ void meta_scan(BrickMeta &mt, int nrows) {
  int acc = 0;
  for (int r = 0; r < nrows; r++) {
    const int c = mt.rstart[r];
    mt.rstart[r] = acc;
    acc += c;
  }
  mt.rstart[nrows] = acc;
  mt.total = acc;
}

// barrier of one group (named barrier `id`, `count` threads) that also ORs a flag over the group
__device__ __forceinline__ bool group_any(int id, int count, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(count)
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(kFgThreads, 1) k_force_gather(PM3K p, int mc, int64_t nbricks,
                                                                const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) float fg_smem[];
  // the tensor copies land on a 128-byte aligned shared address
  float *pot = fg_smem + ((128u - (smem_addr(fg_smem) & 127u)) & 127u) / 4;  // [z 22][y 22][x 24]
  float *fwb = pot + kPotElems;                                                 // [2][3][z][y][x] 18^3
  __shared__ __align__(8) uint64_t bar_pot, bar_full[2], bar_empty[2];
  __shared__ BrickMeta meta[2];
  __shared__ BrickPos s_next;     // the producers' next brick
  __shared__ int64_t s_next_id;   // its index (>= nbricks: none)
  __shared__ float red[4][kFgThreads / 32];
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  const int cb = kBrick / mc, nrows = cb * cb;
  const int64_t n = p.n;
  const bool producer = tid < kFgProd;
  const int gt = producer ? tid : tid - kFgProd;  // thread index in the group
  const int lane = tid & 31;
  if (blockIdx.x >= nbricks) return;
  auto request = [&](const BrickPos &q) {  // thread 0: the potential window of brick q
    mbar_arrive_expect_tx(&bar_pot, kPotBytes);  // the phase completes when the bytes have landed
    const int cx = (int)q.X0 - 4 + kPotPad, cy = (int)q.Y0 - 3 + kPotPad, cz = (int)q.Z0 - 3 + kPotPad;
    const int cs = p.jobs[q.j].slot;
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(pot)),
        "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(cx), "r"(cy), "r"(cz), "r"(cs), "r"(smem_addr(&bar_pot))
        : "memory");
  };
  if (tid == 0) {
    mbar_init(&bar_pot, 1);
    for (int b = 0; b < 2; b++) {
      mbar_init(&bar_full[b], kFgProd / 32);
      mbar_init(&bar_empty[b], kFgCons / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
    s_next_id = blockIdx.x;
    s_next = brick_pos(p, blockIdx.x, cb, p.ract, nullptr);
    request(s_next);
  }
  __syncthreads();
  const FDW w;
  float m = 0.f, vm0 = 0.f, vm1 = 0.f, vm2 = 0.f;
  int nreq = 1;  // tensor copies requested (thread 0)
  int nok = 0;   // tensor copies waited for: the next one completes phase nok & 1 of bar_pot
  if (producer) {
    for (int k = 0;; k++) {
      const int b = k & 1;
      float *fw = fwb + b * 3 * kFor3;
      BrickMeta &mt = meta[b];
      // the consumers are done with buffer b (brick k - 2)
      bool bad = k >= 2 && !mbar_wait_bounded(&bar_empty[b], (uint32_t)((k - 2) >> 1) & 1u);
      const bool stop = group_any(1, kFgProd, bad);
      const int64_t id = s_next_id;  // thread 0 wrote it before the barrier above
      if (stop || id >= nbricks) {
        // no more bricks (or a wait gave up): the consumers stop at this buffer
        if (gt == 0) {
          mt.total = -1;
          if (bad) s_fail = 1;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&bar_full[b]);
        break;
      }
      if (gt == 0) mt.pos = s_next;
      group_any(1, kFgProd, false);  // mt.pos visible to the group
      if (gt < nrows) meta_row(p, cb, mt, gt);
      // this brick's potential window
      bad = !mbar_wait_bounded(&bar_pot, (uint32_t)nok & 1u);
      if (!bad) nok++;
      if (group_any(1, kFgProd, bad)) {
        if (gt == 0) {
          mt.total = -1;
          s_fail = 1;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&bar_full[b]);
        break;
      }
      constexpr int PY = kPotX, PZ = kPotX * kPotW;
      for (int e = gt; e < kFor3; e += kFgProd) {
        const int x = e % kForW, y = (e / kForW) % kForW, z = e / (kForW * kForW);
        const int c = (z + 2) * PZ + (y + 2) * PY + (x + 3);
        const float fx = w(pot[c - 2], pot[c - 1], pot[c + 1], pot[c + 2]);
        const float fy = w(pot[c - 2 * PY], pot[c - PY], pot[c + PY], pot[c + 2 * PY]);
        const float fz = w(pot[c - 2 * PZ], pot[c - PZ], pot[c + PZ], pot[c + 2 * PZ]);
        fw[e] = fx;
        fw[kFor3 + e] = fy;
        fw[2 * kFor3 + e] = fz;
        if (x >= 1 && x <= kBrick && y >= 1 && y <= kBrick && z >= 1 && z <= kBrick)
          m = fmaxf(m, fx * fx + fy * fy + fz * fz);
      }
      group_any(1, kFgProd, false);  // the window is read, the force buffer and the row counts written
      if (gt == 0) {
        meta_scan(mt, nrows);
        // claim and request the next brick (the window buffer is free)
        const int64_t nid = gridDim.x + atomicAdd(p.brick_ctr, 1);
        s_next_id = nid;
        if (nid < nbricks) {
          s_next = brick_pos(p, nid, cb, p.ract, nullptr);
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          request(s_next);
          nreq++;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&bar_full[b]);
    }
    // a tensor copy still in flight (a wait gave up) lands before the block's memory is released
    if (gt == 0 && nreq > nok) (void)mbar_wait_bounded(&bar_pot, (uint32_t)nok & 1u);
  } else {
    for (int k = 0;; k++) {
      const int b = k & 1;
      const float *fw = fwb + b * 3 * kFor3;
      const bool bad = !mbar_wait_bounded(&bar_full[b], (uint32_t)(k >> 1) & 1u);
      if (group_any(2, kFgCons, bad)) {
        if (gt == 0) s_fail = 1;
        break;
      }
      const BrickMeta &mt = meta[b];
      if (mt.total < 0) break;
      const BrickPos &q = mt.pos;
      const MeshJob &J = p.jobs[q.j];
      BrickRows br;
      br.nrows = nrows;
      br.total = mt.total;
      br.cb = cb;
      for (int kk = gt; kk < br.total; kk += kFgCons) {
        int di, dj, dk;
        const int64_t ip = brick_particle(kk, br, mt.rbase, mt.rstart, mt.rcell, di, dj, dk);
        const int16_t *qp = p.xp + 3 * ip;
        float wx[3], wy[3], wz[3];
        const int64_t ix = tsc(decode_pos(q.ci0 + di - p.ncb, qp[0]) * p.scale - J.off[0], wx) + p.shift;
        const int64_t iy = tsc(decode_pos(q.cj0 + dj - p.ncb, qp[1]) * p.scale - J.off[1], wy) + p.shift;
        const int64_t iz = tsc(decode_pos(q.ck0 + dk - p.ncb, qp[2]) * p.scale - J.off[2], wz) + p.shift;
        // the stencil's first point ix - 1 lies at force-window index ix - X0
        const int lx = (int)wrap_near(ix - q.X0, n), ly = (int)wrap_near(iy - q.Y0, n),
                  lz = (int)wrap_near(iz - q.Z0, n);
        float d0 = 0.f, d1 = 0.f, d2 = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
#pragma unroll
          for (int bb = 0; bb < 3; bb++) {
            const int row = ((lz + c) * kForW + (ly + bb)) * kForW + lx;
#pragma unroll
            for (int a = 0; a < 3; a++) {
              const float wt = (wx[a] * wy[bb]) * wz[c];
              d0 += fw[row + a] * wt;
              d1 += fw[kFor3 + row + a] * wt;
              d2 += fw[2 * kFor3 + row + a] * wt;
            }
          }
        }
        float *v = p.vp + 3 * ip;
        const float v0 = v[0] + d0 * p.kick, v1 = v[1] + d1 * p.kick, v2 = v[2] + d2 * p.kick;
        v[0] = v0;
        v[1] = v1;
        v[2] = v2;
        vm0 = fmaxf(vm0, fabsf(v0));
        vm1 = fmaxf(vm1, fabsf(v1));
        vm2 = fmaxf(vm2, fabsf(v2));
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&bar_empty[b]);
    }
  }
  __syncthreads();
  if (tid == 0 && s_fail && p.err) atomicOr(p.err, 1 << CUBE_ERR_TIMEOUT);
  // one update of each maximum per block
  const int warp = tid >> 5;
  m = warp_max(m);
  vm0 = warp_max(vm0);
  vm1 = warp_max(vm1);
  vm2 = warp_max(vm2);
  if (lane == 0) {
    red[0][warp] = m;
    red[1][warp] = vm0;
    red[2][warp] = vm1;
    red[3][warp] = vm2;
  }
  __syncthreads();
  if (tid < 4) {
    float r = 0.f;
    for (int qq = 0; qq < kFgThreads / 32; qq++) r = fmaxf(r, red[tid][qq]);
    if (tid == 0) atomic_max_nonneg(&p.out[0], r);
    else if (p.want_vmax) atomic_max_nonneg(&p.out[1 + tid], r);
  }
}

static PM3K make_k(const PM3Args &a) {
  const Lay &L = *a.L;
  PM3K p;
  p.n = a.n;
  p.nt = L.nt;
  p.nte = L.nte;
  p.ncb = L.ncb;
  p.n3 = (int64_t)a.n * a.n * a.n;
  p.nk = (int64_t)a.n * a.n * (a.n / 2 + 1);
  for (int d = 0; d < 3; d++) {
    p.rdep[d] = a.rdep[d];
    p.ract[d] = a.ract[d];
  }
  p.wrap = a.wrap;
  p.shift = a.shift;
  p.scale = a.scale;
  p.jobs = a.jobs;
  p.njobs = a.njobs;
  p.xp = a.xp;
  p.rhoc = a.rhoc;
  p.cell_base = a.cell_base;
  p.rho = a.rho;
  p.rhok = a.rhok;
  p.force = a.force;
  p.green = a.green;
  p.gscale = (float)((double)a.mass / ((double)a.n * a.n * a.n));
  p.kick = a.kick;
  p.vp = a.vp;
  p.out = a.out;
  p.want_vmax = a.want_vmax;
  p.fphys_lo = a.fphys_lo;
  p.fphys_n = a.fphys_n;
  p.nslots = a.nslots;
  p.err = a.err;
  p.brick_ctr = a.brick_ctr;
  return p;
}


void launch_pm3_kspace(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  k_kspace<<<148 * 8, 256, 0, s>>>(p);
}

// ---------------------------------------------------------------------------------------------
// k-space step fused along z.  After two-dimensional R2C transforms of the x-y planes, the
// half-spectrum is laid out [z][ky][kx] (kx < n/2 + 1); every (kx, ky) column is transformed
// along z, multiplied by the Green table (real), and transformed back, in one read and one write
// of the spectrum (the three-dimensional path reads and writes it three times for the same:
// the last forward pass, the k-space multiply and the first inverse pass).  The two-dimensional
// C2R transforms of the planes then finish the inverse.
//
// The z transforms are iterative Stockham radix-8 FFTs in shared memory (Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors", SC 2008), with a
// radix-4 or radix-2 last pass for lengths that are not powers of 8; twiddles exp(-2 pi i k/N)
// are rounded from double precision.  The inverse runs as the forward transform of the complex
// conjugate (G is real): conj(FFT(conj(X) G)).  Unnormalised, like cuFFT.
constexpr int kZThreads = 512;
constexpr int kZRows = 4;  // ky rows per block (the twiddle table is built once per block)

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)

// 8-point DFT in place (decimation in frequency: radix-2 passes, outputs put back in order)
__device__ __forceinline__ void dft8(float2 v[8]) {
  constexpr float h = 0.70710678118654752f;  // sqrt(2) / 2
  float2 a[8];
  for (int k = 0; k < 4; k++) {
    a[k] = cadd(v[k], v[k + 4]);
    a[k + 4] = csub(v[k], v[k + 4]);
  }
  a[5] = make_float2(h * (a[5].x + a[5].y), h * (a[5].y - a[5].x));    // * exp(-i pi/4)
  a[6] = mul_mi(a[6]);                                                 // * exp(-i pi/2)
  a[7] = make_float2(h * (a[7].y - a[7].x), -h * (a[7].x + a[7].y));   // * exp(-3i pi/4)
  float2 b[8];
  for (int q = 0; q < 8; q += 4) {
    b[q] = cadd(a[q], a[q + 2]);
    b[q + 2] = csub(a[q], a[q + 2]);
    b[q + 1] = cadd(a[q + 1], a[q + 3]);
    b[q + 3] = mul_mi(csub(a[q + 1], a[q + 3]));
  }
  v[0] = cadd(b[0], b[1]);
  v[4] = csub(b[0], b[1]);
  v[2] = cadd(b[2], b[3]);
  v[6] = csub(b[2], b[3]);
  v[1] = cadd(b[4], b[5]);
  v[5] = csub(b[4], b[5]);
  v[3] = cadd(b[6], b[7]);
  v[7] = csub(b[6], b[7]);
}

// One Stockham pass of radix R over the TX columns in s[z * TX + c]: butterfly j of column c
// reads points j + r N/R, applies the twiddles of its position k = j mod Ns and writes the
// R outputs to (j / Ns) Ns R + k + r Ns.
template <int N, int TX, int R, int Ns, int T>
__device__ __forceinline__ void stockham_pass(float2 *s, const float2 *w) {
  constexpr int kButterflies = N / R, kPer = kButterflies * TX / T;  // per thread
  float2 v[kPer][R];
  int dst[kPer];
  const int c = threadIdx.x % TX;
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int j = threadIdx.x / TX + u * (T / TX);
    const int k = j % Ns;
#pragma unroll
    for (int r = 0; r < R; r++) v[u][r] = s[(j + r * kButterflies) * TX + c];
#pragma unroll
    for (int r = 1; r < R; r++) v[u][r] = cmul(v[u][r], w[r * k * (N / (Ns * R))]);
    if (R == 8) {
      dft8(v[u]);
    } else if (R == 4) {
      const float2 a0 = cadd(v[u][0], v[u][2]), a2 = csub(v[u][0], v[u][2]), a1 = cadd(v[u][1], v[u][3]),
                   a3 = mul_mi(csub(v[u][1], v[u][3]));
      v[u][0] = cadd(a0, a1);
      v[u][2] = csub(a0, a1);
      v[u][1] = cadd(a2, a3);
      v[u][3] = csub(a2, a3);
    } else {
      const float2 t = v[u][1];
      v[u][1] = csub(v[u][0], t);
      v[u][0] = cadd(v[u][0], t);
    }
    dst[u] = (j / Ns) * Ns * R + k;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < kPer; u++)
#pragma unroll
    for (int r = 0; r < R; r++) s[(dst[u] + r * Ns) * TX + c] = v[u][r];
  __syncthreads();
}

// radix-8 passes while 8 Ns divides N, then one radix-4 or radix-2 pass (T threads)
template <int N, int TX, int T, int Ns = 1>
__device__ __forceinline__ void fft_columns(float2 *s, const float2 *w) {
  if constexpr (Ns * 8 <= N) {
    stockham_pass<N, TX, 8, Ns, T>(s, w);
    fft_columns<N, TX, T, Ns * 8>(s, w);
  } else if constexpr (Ns * 4 == N) {
    stockham_pass<N, TX, 4, Ns, T>(s, w);
  } else if constexpr (Ns * 2 == N) {
    stockham_pass<N, TX, 2, Ns, T>(s, w);
  }
}

// threads of the generic kernel: columns of eight points (64-byte rows of the spectrum)
template <int N>
struct ZThreads {
  static constexpr int T = N >= 1024 ? 1024 : kZThreads;
};

template <int N>
__global__ void __launch_bounds__(ZThreads<N>::T, (ZThreads<N>::T == 1024 ? 1 : 3))
    k_kspace_z(float2 *C, const float *G, float gscale) {
  constexpr int T = ZThreads<N>::T;
  constexpr int H = N / 2 + 1, TX = T * 8 / N;
  constexpr int64_t kPlane = (int64_t)N * H;  // z stride of the spectrum
  extern __shared__ float2 zg[];
  float2 *const s = zg, *const w = zg + N * TX;
  for (int k = threadIdx.x; k < N; k += T) {
    double sn, cs;
    sincospi(-2.0 * (double)k / (double)N, &sn, &cs);
    w[k] = make_float2((float)cs, (float)sn);
  }
  const int kx0 = blockIdx.x * TX;
  float2 *slot = C + (int64_t)blockIdx.z * N * kPlane;
  for (int ky = blockIdx.y * kZRows; ky < min((int)(blockIdx.y + 1) * kZRows, N); ky++) {
    float2 *col = slot + (int64_t)ky * H + kx0;
    const float *g = G + (int64_t)ky * H + kx0;
    __syncthreads();  // the previous row's stores have read s; the twiddles are written
    constexpr int kPer = N * TX / T;  // points per thread
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int e = threadIdx.x + u * T, z = e / TX, c = e % TX;
      const bool in = kx0 + c < H;
      s[e] = in ? col[z * kPlane + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_columns<N, TX, T>(s, w);
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int e = threadIdx.x + u * T;
      const int z = e / TX, cc = e % TX;
      const float gs = (kx0 + cc < H ? g[z * kPlane + cc] : 0.f) * gscale;
      s[e] = make_float2(s[e].x * gs, -s[e].y * gs);  // conj(X) G
    }
    __syncthreads();
    fft_columns<N, TX, T>(s, w);
#pragma unroll
    for (int u = 0; u < kPer; u++) {
      const int e = threadIdx.x + u * T, z = e / TX, c = e % TX;
      if (kx0 + c < H) col[z * kPlane + c] = make_float2(s[e].x, -s[e].y);
    }
  }
}

// Mesh sides that are powers of 8 (64, 512): every pass is radix 8, so the first pass of each
// transform reads its eight points straight from registers (loaded from the spectrum, or left
// by the last forward pass: the last pass of a Stockham transform leaves point j + r N/8 with
// butterfly j, which is what the first pass wants) and the last pass keeps its outputs in
// registers; only the passes in between go through shared memory, double-buffered (two
// barriers per transform).  Point z of column c sits in shared row z xor (bit 3 of z) (a
// permutation of the rows), which spreads the first pass's stores over all banks for TX = 8.
template <int N>
struct Pow8 {
  static constexpr int P = N == 64 ? 2 : (N == 512 ? 3 : 0);
};
template <int TX>
__device__ __forceinline__ int zpos(int z, int c) {
  return (z ^ ((z >> 3) & 1)) * TX + c;
}

// Radix-8 pass Ns of butterfly j on v (twiddles, then the 8-point DFT)
template <int N, int Ns>
__device__ __forceinline__ void r8_pass(float2 v[8], const float2 *w, int j) {
  if constexpr (Ns > 1) {
    const int k = j % Ns;
#pragma unroll
    for (int r = 1; r < 8; r++) v[r] = cmul(v[r], w[r * k * (N / (Ns * 8))]);
  }
  dft8(v);
}
template <int N, int TX, int Ns>
__device__ __forceinline__ void r8_store(float2 *buf, const float2 v[8], int j, int c) {
  const int d = (j / Ns) * Ns * 8 + j % Ns;
#pragma unroll
  for (int r = 0; r < 8; r++) buf[zpos<TX>(d + r * Ns, c)] = v[r];
}
template <int N, int TX>
__device__ __forceinline__ void r8_load(const float2 *buf, float2 v[8], int j, int c) {
#pragma unroll
  for (int r = 0; r < 8; r++) v[r] = buf[zpos<TX>(j + r * (N / 8), c)];
}
// the transform of v (point j + r N/8 of column c), result in v at the same points.  Three
// passes store to sa then sb and read them in that order; two passes store to and read sa.
template <int N, int TX>
__device__ __forceinline__ void fft8_regs(float2 v[8], float2 *sa, float2 *sb, const float2 *w, int j, int c) {
  r8_pass<N, 1>(v, w, j);
  r8_store<N, TX, 1>(sa, v, j, c);
  __syncthreads();
  r8_load<N, TX>(sa, v, j, c);
  if constexpr (Pow8<N>::P == 3) {
    r8_pass<N, 8>(v, w, j);
    r8_store<N, TX, 8>(sb, v, j, c);
    __syncthreads();
    r8_load<N, TX>(sb, v, j, c);
    r8_pass<N, 64>(v, w, j);
  } else {
    r8_pass<N, 8>(v, w, j);
  }
}

template <int N>
__global__ void __launch_bounds__(kZThreads, 2) k_kspace_z8(float2 *C, const float *G, float gscale) {
  constexpr int H = N / 2 + 1, TX = kZThreads * 8 / N;
  constexpr int64_t kPlane = (int64_t)N * H;
  constexpr int kBuf = N * TX;
  extern __shared__ float2 zs[];
  float2 *const sa = zs, *const sb = zs + kBuf, *const w = zs + 2 * kBuf;
  for (int k = threadIdx.x; k < N; k += kZThreads) {
    double sn, cs;
    sincospi(-2.0 * (double)k / (double)N, &sn, &cs);
    w[k] = make_float2((float)cs, (float)sn);
  }
  __syncthreads();
  const int c = threadIdx.x % TX, j = threadIdx.x / TX, kx0 = blockIdx.x * TX;
  const bool in = kx0 + c < H;
  float2 *slot = C + (int64_t)blockIdx.z * N * kPlane;
  for (int ky = blockIdx.y * kZRows; ky < min((int)(blockIdx.y + 1) * kZRows, N); ky++) {
    float2 *col = slot + (int64_t)ky * H + kx0 + c;
    const float *g = G + (int64_t)ky * H + kx0 + c;
    float2 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) v[r] = in ? col[(j + r * (N / 8)) * kPlane] : make_float2(0.f, 0.f);
    fft8_regs<N, TX>(v, sa, sb, w, j, c);  // last read: sb (three passes) or sa (two)
#pragma unroll
    for (int r = 0; r < 8; r++) {  // conj(X) G
      const float gs = (in ? g[(j + r * (N / 8)) * kPlane] : 0.f) * gscale;
      v[r] = make_float2(v[r].x * gs, -v[r].y * gs);
    }
    // the inverse's first store goes to the buffer that no thread may still be reading
    if constexpr (Pow8<N>::P == 3) fft8_regs<N, TX>(v, sa, sb, w, j, c);
    else fft8_regs<N, TX>(v, sb, sa, w, j, c);
    if (in) {
#pragma unroll
      for (int r = 0; r < 8; r++) col[(j + r * (N / 8)) * kPlane] = make_float2(v[r].x, -v[r].y);
    }
  }
}
constexpr size_t kz8_smem(int n) { return sizeof(float2) * (2 * (size_t)(n * (kZThreads * 8 / n)) + n); }

// Mesh sides that take the fused z step
bool pm3_kspace_z_ok(int n) { return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024; }

static void set_smem_attr_once(const void *fn, size_t bytes);

template <int N>
static void launch_kz(const PM3K &p, cudaStream_t s) {
  if constexpr (Pow8<N>::P > 0) {
    constexpr int TX = kZThreads * 8 / N;
    const dim3 grid((unsigned)((N / 2 + 1 + TX - 1) / TX), (unsigned)((N + kZRows - 1) / kZRows), (unsigned)p.nslots);
    constexpr size_t smem = kz8_smem(N);
    set_smem_attr_once((const void *)k_kspace_z8<N>, smem);
    k_kspace_z8<N><<<grid, kZThreads, smem, s>>>(p.rhok, p.green, p.gscale);
  } else {
    constexpr int T = ZThreads<N>::T, TX = T * 8 / N;
    const dim3 grid((unsigned)((N / 2 + 1 + TX - 1) / TX), (unsigned)((N + kZRows - 1) / kZRows), (unsigned)p.nslots);
    constexpr size_t smem = sizeof(float2) * (size_t)(N * TX + N);
    set_smem_attr_once((const void *)k_kspace_z<N>, smem);
    k_kspace_z<N><<<grid, T, smem, s>>>(p.rhok, p.green, p.gscale);
  }
}

void launch_pm3_kspace_z(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  switch (a.n) {
    case 64: launch_kz<64>(p, s); break;
    case 128: launch_kz<128>(p, s); break;
    case 256: launch_kz<256>(p, s); break;
    case 512: launch_kz<512>(p, s); break;
    case 1024: launch_kz<1024>(p, s); break;
    default: break;  // other sides take the three-dimensional path (pm3_kspace_z_ok)
  }
}

void launch_pm3_force(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  if (a.n % 4 == 0) {
    const int nzc = (a.n + kFzChunk - 1) / kFzChunk;
    const dim3 grid((unsigned)((a.n / 4 + 31) / 32), (unsigned)((a.n + kFzRows - 1) / kFzRows),
                    (unsigned)(nzc * a.nslots));
    k_force_zm<<<grid, kFzRows * 32, 0, s>>>(p);
  } else
    k_force<<<148 * 8, 256, 0, s>>>(p);
}

// Deposit brick by brick: the TSC weights of the brick's particles accumulate in a shared-memory
// window (the brick plus one point on every side, widened to whole 16-byte groups along x) with
// native 32-bit integer shared atomics on fixed-point weights, w * 2^e rounded to an integer; e
// is chosen per brick from its particle count so that no window point can overflow 2^32
// (a point takes at most 0.75^3 of each particle).  The window then goes to the mesh as floats,
// one 16-byte vector reduction per group of four points that received anything: every mesh point
// takes at most one global reduction per brick that reaches it, instead of one per particle.
// kick.f90:420-468 sums the same weights; the integer sums make the brick's part exact and
// independent of the order of the atomics (the rounding of a weight to 2^-e, e >= 15 for
// bricks of up to 10^5 particles, is far below the FP32 rounding of the density).
constexpr int kDepThreads = 256;
constexpr int kAccX = kBrick + 8;  // x window owned - 4 .. owned + kBrick + 3: whole float4 groups
constexpr int kAccW = kBrick + 2;  // y, z window owned - 1 .. owned + kBrick

constexpr int kDepChunk = 2048;  // particles of one deposit work item (a crowded brick makes several)

// The deposit's work list: every brick with particles makes ceil(particles / kDepChunk) items
// (brick, chunk, chunks), so a crowded brick is spread over several blocks whose windows add up
// in the mesh; empty bricks make none.  One thread per brick; items[0..count) in any order.
__global__ void k_dep_items(PM3K p, int mc, int64_t nbricks, int chunk, int2 *items, int *count, int64_t cap) {
  const int cb = kBrick / mc;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nbricks;
       b += (int64_t)gridDim.x * blockDim.x) {
    const BrickPos q = brick_pos(p, b, cb, p.rdep, p.rdep);
    const int64_t t = p.jobs[q.j].t;
    int total = 0;
    for (int k = 0; k < cb; k++)
      for (int j = 0; j < cb; j++) {
        const int32_t *r = p.rhoc + ((t * p.nte + q.ck0 + k) * p.nte + q.cj0 + j) * p.nte + q.ci0;
        for (int i = 0; i < cb; i++) total += r[i];
      }
    if (total == 0) continue;
    const int nch = min((total + chunk - 1) / chunk, 0x7fff);
    const int at = atomicAdd(count, nch);
    if (at + nch > cap) {  // more particles in the cells than stored: the cell counts are wrong
      if (p.err) atomicOr(p.err, 1 << CUBE_ERR_CAPACITY);
      continue;
    }
    for (int c = 0; c < nch; c++) items[at + c] = make_int2((int)b, c | (nch << 16));
  }
}

__global__ void __launch_bounds__(kDepThreads) k_deposit_brick(PM3K p, int mc, const int2 *items, const int *count) {
  __shared__ __align__(16) unsigned acc[kAccW * kAccW * kAccX];
  __shared__ int64_t rbase[kMaxRowsPerBrick];
  __shared__ int rstart[kMaxRowsPerBrick + 1];
  __shared__ int rcell[kMaxRowsPerBrick * (kMaxCb + 1)];
  int2 item = make_int2((int)blockIdx.x, 1 << 16);  // without a work list: one block per whole brick
  if (items) {
    if ((int)blockIdx.x >= min(*count, (int)gridDim.x)) return;
    item = items[blockIdx.x];
  }
  const int chunk = item.y & 0xffff, nch = item.y >> 16;
  const int cb = kBrick / mc;
  const BrickPos q = brick_pos(p, item.x, cb, p.rdep, p.rdep);
  const MeshJob &J = p.jobs[q.j];
  const int64_t n = p.n;
  for (int e4 = threadIdx.x; e4 < kAccW * kAccW * kAccX / 4; e4 += kDepThreads)
    reinterpret_cast<uint4 *>(acc)[e4] = make_uint4(0u, 0u, 0u, 0u);
  BrickRows br;
  brick_rows(p, J, cb, q.ci0, q.cj0, q.ck0, rbase, rstart, rcell, br);  // its barriers cover the zeroing
  // this item's particles of the brick
  const int k0 = (int)((int64_t)br.total * chunk / nch), k1 = (int)((int64_t)br.total * (chunk + 1) / nch);
  if (k1 <= k0) return;
  // fixed-point scale 2^e: particles * 0.4219 * 2^e < 2^32
  int e = 24;
  while (e > 1 && (double)(k1 - k0) * 0.421875 * (double)(1u << e) >= 4294967040.0) e--;
  const float fs = (float)(1u << e), inv = 1.0f / fs;
  for (int k = k0 + threadIdx.x; k < k1; k += kDepThreads) {
    int di, dj, dk;
    const int64_t ip = brick_particle(k, br, rbase, rstart, rcell, di, dj, dk);
    const int16_t *qp = p.xp + 3 * ip;
    float wx[3], wy[3], wz[3];
    const int64_t ix = tsc(decode_pos(q.ci0 + di - p.ncb, qp[0]) * p.scale - J.off[0], wx) + p.shift;
    const int64_t iy = tsc(decode_pos(q.cj0 + dj - p.ncb, qp[1]) * p.scale - J.off[1], wy) + p.shift;
    const int64_t iz = tsc(decode_pos(q.ck0 + dk - p.ncb, qp[2]) * p.scale - J.off[2], wz) + p.shift;
    // window indices of the stencil's first point: x (ix - 1) - (X0 - 4), y (iy - 1) - (Y0 - 1)
    const int lx = (int)wrap_near(ix - q.X0, n) + 3, ly = (int)wrap_near(iy - q.Y0, n),
              lz = (int)wrap_near(iz - q.Z0, n);
    const float sx0 = wx[0] * fs, sx1 = wx[1] * fs, sx2 = wx[2] * fs;
#pragma unroll
    for (int c = 0; c < 3; c++) {
#pragma unroll
      for (int bb = 0; bb < 3; bb++) {
        unsigned *row = acc + ((lz + c) * kAccW + (ly + bb)) * kAccX + lx;
        const float yz = wy[bb] * wz[c];
        atomicAdd(row + 0, __float2uint_rn(sx0 * yz));
        atomicAdd(row + 1, __float2uint_rn(sx1 * yz));
        atomicAdd(row + 2, __float2uint_rn(sx2 * yz));
      }
    }
  }
  __syncthreads();
  // Flush: lane (w, xg) of a warp takes x group xg (lane % 6) of window rows 5 pass + w (w < 5), so
  // the group's mesh x index is worked out once and each row's once per pass.
  float *R = p.rho + (int64_t)J.slot * p.n3;
  constexpr int G4 = kAccX / 4, kRowsPerWarp = 32 / G4, kRows = kAccW * kAccW;
  const int lane = threadIdx.x & 31, w = lane / G4, xg = lane - w * G4;
  if (w < kRowsPerWarp) {
    const int ni = (int)n;
    auto wrap32 = [ni](int a) { return a < 0 ? a + ni : (a >= ni ? a - ni : a); };
    const int gx = wrap32((int)q.X0 - 4 + 4 * xg);
    for (int row = (threadIdx.x >> 5) * kRowsPerWarp + w; row < kRows; row += (kDepThreads / 32) * kRowsPerWarp) {
      const uint4 u = reinterpret_cast<const uint4 *>(acc)[row * G4 + xg];
      if ((u.x | u.y | u.z | u.w) == 0u) continue;
      const int gy = wrap32((int)q.Y0 - 1 + row % kAccW), gz = wrap32((int)q.Z0 - 1 + row / kAccW);
      atomicAdd(reinterpret_cast<float4 *>(R + ((int64_t)gz * ni + gy) * ni + gx),
                make_float4((float)u.x * inv, (float)u.y * inv, (float)u.z * inv, (float)u.w * inv));
    }
  }
}

// mesh points per coarse cell when the brick kernels apply (periodic meshes, whole mesh points
// per coarse cell dividing the brick, the deposited (dep) or gathered cells of every job a whole
// number of bricks), else 0
static int brick_mc(const PM3Args &a, bool dep) {
  if (!a.wrap || a.n < 8) return 0;
  const double mcd = a.scale;
  const int mc = (int)llrint(mcd);
  if (mc < 1 || (double)mc != mcd || kBrick % mc) return 0;
  const int cb = kBrick / mc;
  if (cb > kMaxCb) return 0;
  for (int d = 0; d < 3; d++)
    if ((dep ? a.rdep[d] : a.ract[d]) % cb) return 0;
  return mc;
}
int pm3_brick_mc(const PM3Args &a) { return brick_mc(a, false); }

// the dynamic shared-memory limit of a kernel, raised once per device (the attribute is per device)
static void set_smem_attr_once(const void *fn, size_t bytes) {
  constexpr int kDev = 64, kFn = 16;
  static const void *fns[kFn] = {};
  static bool done[kFn][kDev] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int f = 0;
  while (f < kFn && fns[f] && fns[f] != fn) f++;
  if (f == kFn) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return;
  }
  fns[f] = fn;
  if (dev >= 0 && dev < kDev && done[f][dev]) return;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (dev >= 0 && dev < kDev) done[f][dev] = true;
}

size_t pm3_dep_items_bytes(int64_t cells_per_job, int njobs, int64_t n_used) {
  // bricks hold at least one coarse cell: one item per cell, plus one per kDepChunk particles, plus the count
  return sizeof(int2) * ((size_t)cells_per_job * njobs + (size_t)(n_used / kDepChunk) + 2);
}

int launch_pm3_deposit(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  const int mc = (a.n % 4 == 0) ? brick_mc(a, true) : 0;
  if (mc) {
    constexpr int chunk = kDepChunk;
    auto kern = k_deposit_brick;
    const int cb = kBrick / mc;
    const int64_t nbricks = (int64_t)(a.rdep[0] / cb) * (a.rdep[1] / cb) * (a.rdep[2] / cb) * a.njobs;
    if (nbricks <= 0) return 0;
    if (!a.dep_items) {
      kern<<<(unsigned)nbricks, kDepThreads, 0, s>>>(p, mc, nullptr, nullptr);
      return 1;
    }
    // at most one item per brick plus one per `chunk` particles
    const int64_t cap = nbricks + a.n_particles_hint / chunk + 1;
    int *count = reinterpret_cast<int *>(a.dep_items + cap);
    cudaMemsetAsync(count, 0, sizeof(int), s);
    k_dep_items<<<(unsigned)std::min<int64_t>((nbricks + 255) / 256, 4096), 256, 0, s>>>(p, mc, nbricks, chunk,
                                                                                       a.dep_items, count, cap);
    kern<<<(unsigned)cap, kDepThreads, 0, s>>>(p, mc, a.dep_items, count);
    return 2;
  }
  const int64_t warps = (int64_t)a.rdep[0] * a.rdep[1] * a.rdep[2] * a.njobs;
  k_deposit<<<(unsigned)((warps + kWarps - 1) / kWarps), kWarps * 32, 0, s>>>(p);
  return 1;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
  }
  return fn;
}

bool launch_pm3_force_gather(const PM3Args &a, cudaStream_t s) {
  const int mc = brick_mc(a, false);
  if (!mc || !a.phi_pad) return false;
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return false;
  // the padded potential as a 4-d tensor [slot][z][y][x], boxes of the potential window
  const cuuint64_t m = (cuuint64_t)a.n + 2 * kPotPad;
  const cuuint64_t dims[4] = {m, m, m, (cuuint64_t)a.nslots};
  const cuuint64_t strides[3] = {m * 4, m * m * 4, m * m * m * 4};
  const cuuint32_t box[4] = {kPotX, kPotW, kPotW, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap tmap;
  if (encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.phi_pad, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  PM3K p = make_k(a);
  const int cb = kBrick / mc;
  const int64_t nbricks = (int64_t)(a.ract[0] / cb) * (a.ract[1] / cb) * (a.ract[2] / cb) * a.njobs;
  set_smem_attr_once((const void *)k_force_gather, kFgSmem);
  const int64_t grid = std::min<int64_t>(nbricks, a.num_sms > 0 ? a.num_sms : 148);
  if (!a.brick_ctr) return false;
  cudaMemsetAsync(a.brick_ctr, 0, sizeof(int32_t), s);
  if (grid > 0) k_force_gather<<<(unsigned)grid, kFgThreads, kFgSmem, s>>>(p, mc, nbricks, tmap);
  return true;
}

// ghost points of the padded potential: each takes the interior point it is a periodic image of.
// The z slabs (all y, x), the y slabs (interior z, all x) and the x slabs (interior z, y) are
// disjoint and together cover every ghost point once.
__global__ void k_pm3_ghosts(float *phi, int n, int nslots) {
  const int P = kPotPad;
  const int m = n + 2 * P;
  const int nz = 2 * P * m * m, ny = n * 2 * P * m, nx = n * n * 2 * P;
  const int per = nz + ny + nx;
  const int sl = blockIdx.y;
  float *base = phi + (int64_t)sl * m * m * m;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < per; e += gridDim.x * blockDim.x) {
    int r = e, x, y, z;
    if (r < nz) {
      x = r % m;
      y = (r / m) % m;
      const int g = r / (m * m);  // 0 .. 2P-1
      z = g < P ? g : n + g;
    } else if ((r -= nz) < ny) {
      x = r % m;
      const int g = (r / m) % (2 * P);
      y = g < P ? g : n + g;
      z = P + r / (m * 2 * P);
    } else {
      r -= ny;
      const int g = r % (2 * P);
      x = g < P ? g : n + g;
      y = P + (r / (2 * P)) % n;
      z = P + r / (2 * P * n);
    }
    const int sx = x < P ? x + n : (x >= n + P ? x - n : x);
    const int sy = y < P ? y + n : (y >= n + P ? y - n : y);
    const int sz = z < P ? z + n : (z >= n + P ? z - n : z);
    base[((int64_t)z * m + y) * m + x] = base[((int64_t)sz * m + sy) * m + sx];
  }
}

void launch_pm3_ghosts(const PM3Args &a, cudaStream_t s) {
  if (!a.phi_pad) return;
  const int m = a.n + 2 * kPotPad;
  const int64_t per = (int64_t)2 * kPotPad * m * m + (int64_t)a.n * 2 * kPotPad * m + (int64_t)a.n * a.n * 2 * kPotPad;
  const unsigned gx = (unsigned)std::min<int64_t>((per + 255) / 256, 4096);
  k_pm3_ghosts<<<dim3(gx, (unsigned)a.nslots), 256, 0, s>>>(a.phi_pad, a.n, a.nslots);
}

void launch_pm3_gather(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  const int64_t warps = (int64_t)a.ract[0] * a.ract[1] * a.ract[2] * a.njobs;
  k_gather<<<(unsigned)((warps + kWarps - 1) / kWarps), kWarps * 32, 0, s>>>(p);
}

// ---------------------------------------------------------------------------------------------
// Green_3D (Green/Green.f90:1-80) in FP64 on the device.  G depends on |k_d|
// per axis only, so one thread evaluates an octant point and writes its (up
// to) four mirror images in the stored half spectrum [k3][k2][k1].

struct GreenK {
  int n;
  double apm_soft, apm_range, gpow, alpha, c215;
  int p2;  // 2p+2
  const double *fs;
  float *G;
};

__global__ void k_green(GreenK p) {
  const int h = p.n / 2;
  const int64_t tot = (int64_t)(h + 1) * (h + 1) * (h + 1);
  const double twopi = 6.283185307179586476925286766559;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % (h + 1)), b = (int)((e / (h + 1)) % (h + 1)), c = (int)(e / ((int64_t)(h + 1) * (h + 1)));
    const double kv[3] = {p.fs[a], p.fs[b], p.fs[c]};
    double D[3], u2n = 1.0, ur[3] = {0, 0, 0};
    for (int d = 0; d < 3; d++) {
      D[d] = p.alpha * sin(kv[d]) + (1 - p.alpha) * sin(2 * kv[d]) / 2;
      const double s = sin(kv[d] / 2);
      u2n *= 1 - s * s + p.c215 * s * s * s * s;
    }
    for (int i3 = -2; i3 <= 2; i3++)
      for (int i2 = -2; i2 <= 2; i2++)
        for (int i1 = -2; i1 <= 2; i1++) {
          const double kn[3] = {kv[0] + twopi * i1, kv[1] + twopi * i2, kv[2] + twopi * i3};
          const double kmag = sqrt(kn[0] * kn[0] + kn[1] * kn[1] + kn[2] * kn[2]);
          double U = 1.0;
          for (int d = 0; d < 3; d++) U *= (kn[d] == 0.0) ? 1.0 : sin(kn[d] / 2) / (kn[d] / 2);
          double Up = 1.0;
          for (int q = 0; q < p.p2; q++) Up *= U;
          double Ss, Sr;
          if (kmag == 0.0) {
            Ss = 1.0;
          } else {
            const double y = p.apm_soft * kmag / 2;
            double sy, cy;
            sincos(y, &sy, &cy);
            const double y2 = y * y;
            Ss = 12.0 / (y2 * y2) * (2 - 2 * cy - y * sy);
          }
          if (p.apm_range == 0.0) {
            Sr = 0.0;
          } else if (kmag == 0.0) {
            Sr = 1.0;
          } else {
            const double y = p.apm_range * kmag / 2;
            double sy, cy;
            sincos(y, &sy, &cy);
            const double y2 = y * y;
            Sr = 12.0 / (y2 * y2) * (2 - 2 * cy - y * sy);
          }
          const double f = (Ss * Ss - Sr * Sr) / (kmag * kmag);
          for (int d = 0; d < 3; d++) ur[d] += Up * kn[d] * f;
        }
    const double num = D[0] * ur[0] + D[1] * ur[1] + D[2] * ur[2];
    const double den = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
    const double pi4 = 12.566370614359172953850573533118;
    float g = (float)(pi4 * num / den / (u2n * u2n) / p.gpow);
    // Gk(::n/2,::n/2,::n/2) = 0 (Green.f90:71)
    if ((a == 0 || a == h) && (b == 0 || b == h) && (c == 0 || c == h)) g = 0.0f;
    const int n = p.n, nh = h + 1;
    const int bs[2] = {b, (n - b) % n}, cs[2] = {c, (n - c) % n};
    for (int u = 0; u < 2; u++) {
      if (u == 1 && cs[1] == cs[0]) continue;
      for (int v = 0; v < 2; v++) {
        if (v == 1 && bs[1] == bs[0]) continue;
        p.G[((int64_t)cs[u] * n + bs[v]) * nh + a] = g;
      }
    }
  }
}

void launch_green_fp64(int n, double apm_soft, double apm_range, double gridsize, int p_order, float *G,
                       cudaStream_t s) {
  // Fortran literals 4./3, 2./15 and 1./nglobal are single precision, gridsize is real(4)
  double *h_fs = new double[n];
  const double pi = 3.14159265358979323846;
  const double inv_n = (double)(1.0f / (float)n);
  for (int k = 1; k <= n; k++) {
    const int m = (k + n / 2 - 1) % n - n / 2;
    h_fs[k - 1] = 2.0 * pi * inv_n * (double)m;
  }
  double *d_fs = nullptr;
  cudaMallocAsync(&d_fs, sizeof(double) * n, s);
  cudaMemcpyAsync(d_fs, h_fs, sizeof(double) * n, cudaMemcpyHostToDevice, s);
  GreenK p;
  p.n = n;
  p.apm_soft = apm_soft;
  p.apm_range = apm_range;
  const float gs = (float)gridsize;
  p.gpow = (double)(gs * gs);
  p.alpha = (double)(4.0f / 3.0f);
  p.c215 = (double)(2.0f / 15.0f);
  p.p2 = 2 * p_order + 2;
  p.fs = d_fs;
  p.G = G;
  k_green<<<148 * 8, 128, 0, s>>>(p);
  cudaFreeAsync(d_fs, s);
  cudaStreamSynchronize(s);
  delete[] h_fs;
}

}  // namespace cube
