// Per-cell check and fallback of the learned PP shell.  The learned kick (the cutoff-1 split plus
// the network) and the full-cutoff kick (PM3 + PP at cutoff 2, the plain method) of one image
// start from the same velocities; the full-cutoff kick is the reference for the network.  Every
// coarse cell that holds physical particles is checked on its first `samples` particles in storage
// order: the relative rms difference of the two velocity changes over those particles, against
// the bound.  A cell over the bound takes the full-cutoff velocities for all its particles; the
// other cells keep the learned ones.  No reference counterpart (the learned shell is new).
//
// One warp per interior coarse cell (tile, i, j, k): its particles are one contiguous run of
// storage, [idx_b_r(j, k) - sum_{i' >= i} rhoc, + rhoc(i, j, k)) (kick.f90:289).
#include "common.cuh"

namespace cube {

constexpr int kFbWarps = 8;

struct FallbackK {
  Lay L;
  const int32_t *rhoc;
  const int64_t *idx_b_r;
  const float *vp0, *vpl, *vpf;
  float *out;
  float bound2;  // bound^2
  int samples;
  int64_t cells;
  unsigned long long *stats;  // [0] cells checked, [1] cells over the bound, [2] particles fallen back
  double *err;                // [0] sum |dvL - dvF|^2 over the samples, [1] sum |dvF|^2
};

__global__ void __launch_bounds__(kFbWarps * 32) k_learned_fallback(FallbackK p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t c = (int64_t)blockIdx.x * kFbWarps + warp;
  __shared__ unsigned long long s_st[kFbWarps][3];
  __shared__ double s_e[kFbWarps][2];
  unsigned long long checked = 0, over = 0, fell = 0;
  double e_num = 0.0, e_den = 0.0;
  if (c < p.cells) {
    const Lay &L = p.L;
    // c = ((t * nt + k) * nt + j) * nt + i over the interior cells
    const int i = (int)(c % L.nt), j = (int)((c / L.nt) % L.nt), k = (int)((c / ((int64_t)L.nt * L.nt)) % L.nt);
    const int64_t t = c / ((int64_t)L.nt * L.nt * L.nt);
    const int64_t row = (t * L.nte + k + L.ncb) * L.nte + j + L.ncb;
    const int32_t *r = p.rhoc + row * L.nte;
    const int ci = i + L.ncb;
    int tail = 0;  // particles of the row from cell ci on
    for (int q = lane; q < L.nte; q += 32) tail += q >= ci ? r[q] : 0;
    for (int o = 16; o; o >>= 1) tail += __shfl_xor_sync(0xffffffffu, tail, o);
    const int np = r[ci];
    const int64_t base = p.idx_b_r[row] - tail;
    if (np > 0) {
      float num = 0.f, den = 0.f;
      const int ns = min(np, p.samples);
      if (lane < ns) {
        const int64_t q = 3 * (base + lane);
        for (int d = 0; d < 3; d++) {
          const float dl = p.vpl[q + d] - p.vp0[q + d], df = p.vpf[q + d] - p.vp0[q + d];
          num += (dl - df) * (dl - df);
          den += df * df;
        }
      }
      for (int o = 16; o; o >>= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
      }
      const bool bad = num > p.bound2 * den;
      checked = 1;
      over = bad ? 1 : 0;
      fell = bad ? (unsigned long long)np : 0;
      e_num = num;
      e_den = den;
      const float *src = bad ? p.vpf : p.vpl;
      for (int q = lane; q < 3 * np; q += 32) p.out[3 * base + q] = src[3 * base + q];
    }
  }
  if (lane == 0) {
    s_st[warp][0] = checked;
    s_st[warp][1] = over;
    s_st[warp][2] = fell;
    s_e[warp][0] = e_num;
    s_e[warp][1] = e_den;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    unsigned long long v = 0;
    for (int w = 0; w < kFbWarps; w++) v += s_st[w][threadIdx.x];
    if (v) atomicAdd(p.stats + threadIdx.x, v);
  } else if (threadIdx.x < 5) {
    double v = 0.0;
    for (int w = 0; w < kFbWarps; w++) v += s_e[w][threadIdx.x - 3];
    if (v != 0.0) atomicAdd(p.err + threadIdx.x - 3, v);
  }
}

void launch_learned_fallback(const Lay &L, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const float *d_vp0,
                             const float *d_vpl, const float *d_vpf, float bound, int samples, float *d_out,
                             unsigned long long *d_stats, double *d_err, cudaStream_t s) {
  FallbackK p;
  p.L = L;
  p.rhoc = d_rhoc;
  p.idx_b_r = d_idx_b_r;
  p.vp0 = d_vp0;
  p.vpl = d_vpl;
  p.vpf = d_vpf;
  p.out = d_out;
  p.bound2 = bound * bound;
  p.samples = samples;
  p.cells = (int64_t)L.ntile * L.nt * L.nt * L.nt;
  p.stats = d_stats;
  p.err = d_err;
  const int64_t blocks = (p.cells + kFbWarps - 1) / kFbWarps;
  if (blocks > 0) k_learned_fallback<<<(unsigned)blocks, kFbWarps * 32, 0, s>>>(p);
}

}  // namespace cube
