// FP64 conservation sums of a kick: momentum change sum m (vb - va) per axis and kinetic-energy
// change sum m/2 (|vb|^2 - |va|^2) over the physical particles of the image (the interior
// coarse cells of every tile), with sum |m (vb - va)| per axis as their scale.  The reference's
// own run-time invariants are printed sums of the same kind ("sum of PM3 density",
// kick.f90:183; "sum of PP count", kick.f90:230).  The kick itself runs in FP32; only these
// global sums (and the Green table) are FP64.
//
// One warp per interior row (tile, k, j): the row's interior particles are one contiguous run of
// storage, [idx_b_r - sum_{i >= ncb} rhoc, idx_b_r - sum_{i >= ncb + nt} rhoc)
// (kick.f90:289, pp_force_kernel.c:203-209), so the lanes stream it with coalesced loads.  Each
// lane sums in FP64; warps reduce with shuffles, blocks through shared memory, and one FP64
// atomic per block and sum lands in the output.
#include "common.cuh"

namespace cube {

constexpr int kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads) k_kick_sums(Lay L, const int32_t *__restrict__ rhoc,
                                                           const int64_t *__restrict__ idx_b_r,
                                                           const float *__restrict__ va,
                                                           const float *__restrict__ vb, double mass,
                                                           int64_t rows, double *__restrict__ out) {
  __shared__ double red[kSumThreads / 32][kNumKickSums];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc[kNumKickSums];
#pragma unroll
  for (int q = 0; q < kNumKickSums; q++) acc[q] = 0.0;
  const int64_t row = (int64_t)blockIdx.x * (kSumThreads / 32) + warp;
  if (row < rows) {
    // row = (t * nt + kk) * nt + jj over the interior rows; storage row (k, j) = (kk + ncb, jj + ncb)
    const int jj = (int)(row % L.nt), kk = (int)((row / L.nt) % L.nt);
    const int64_t t = row / ((int64_t)L.nt * L.nt);
    const int64_t srow = (t * L.nte + kk + L.ncb) * L.nte + jj + L.ncb;
    const int32_t *r = rhoc + srow * L.nte;
    int tail_in = 0, tail_out = 0;  // sums over i >= ncb and i >= ncb + nt
    for (int i = lane; i < L.nte; i += 32) {
      const int c = r[i];
      tail_in += i >= L.ncb ? c : 0;
      tail_out += i >= L.ncb + L.nt ? c : 0;
    }
    for (int o = 16; o; o >>= 1) {
      tail_in += __shfl_xor_sync(0xffffffffu, tail_in, o);
      tail_out += __shfl_xor_sync(0xffffffffu, tail_out, o);
    }
    const int64_t end = idx_b_r[srow];
    const int64_t lo = end - tail_in, hi = end - tail_out;
    for (int64_t p = lo + lane; p < hi; p += 32) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double a = (double)va[3 * p + d], b = (double)vb[3 * p + d];
        const double dm = mass * (b - a);
        acc[d] += dm;
        acc[4 + d] += fabs(dm);
        acc[3] += 0.5 * mass * (b * b - a * a);
      }
      acc[7] += 1.0;
    }
  }
#pragma unroll
  for (int q = 0; q < kNumKickSums; q++) {
    double v = acc[q];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < kNumKickSums) {
    double v = 0.0;
    for (int w = 0; w < kSumThreads / 32; w++) v += red[w][threadIdx.x];
    if (v != 0.0) atomicAdd(out + threadIdx.x, v);
  }
}

void launch_kick_sums(const Lay &L, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const float *d_va,
                      const float *d_vb, float mass, double *d_out, cudaStream_t s) {
  const int64_t rows = (int64_t)L.ntile * L.nt * L.nt;
  const int64_t blocks = (rows + kSumThreads / 32 - 1) / (kSumThreads / 32);
  if (blocks > 0)
    k_kick_sums<<<(unsigned)blocks, kSumThreads, 0, s>>>(L, d_rhoc, d_idx_b_r, d_va, d_vb, (double)mass, rows,
                                                           d_out);
}

}  // namespace cube
