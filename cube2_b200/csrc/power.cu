// CIC power spectrum of the image's physical particles: the deposit of
// utilities/cicpower.f90:55-70 (cell-centred grid of nw points per side, weights
// (idx1 - x) and (x - idx1 + 1) per axis) and the linear-k binning of
// utilities/powerspectrum.f90:52-94 (cross_power, auto terms): modes of the half spectrum
// without the conjugate duplicates of the i = 0 and i = nyquist planes, bin nint(|k|),
// |delta_k|^2 / sinc^4 (CIC window) and the dimensionless 4 pi k^3 |delta_k|^2 / sinc^4.
// Between the two, delta = rho * nw^3 / N - 1 and one cuFFT R2C (delta_k = FFT / nw^3).
#include "common.cuh"

namespace cube {

struct PowK {
  int nt, ncb, nte, nnt, nc, nw;
  int64_t ncells;  // ntile * nte^3
  int64_t n_used;  // stored copies (bound of the spine)
  const int32_t *rhoc;
  const int64_t *cell_base;
  const int16_t *xp;
  float *grid;     // [nw^3] (z, y, x)
};

// warp per physical coarse cell of a tile
__global__ void __launch_bounds__(256) k_cic_grid(PowK p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n3 = (int64_t)p.nte * p.nte * p.nte;
  const double scale = (double)p.nw / (double)p.nc;
  for (int64_t E = (int64_t)blockIdx.x * 8 + warp; E < p.ncells; E += (int64_t)gridDim.x * 8) {
    const int t = (int)(E / n3);
    int64_t r = E - (int64_t)t * n3;
    const int cz = (int)(r / (p.nte * p.nte));
    r -= (int64_t)cz * p.nte * p.nte;
    const int cy = (int)(r / p.nte), cx = (int)(r - (int64_t)cy * p.nte);
    const int lo = p.ncb, hi = p.ncb + p.nt;
    if (cx < lo || cx >= hi || cy < lo || cy >= hi || cz < lo || cz >= hi) continue;
    const int n = p.rhoc[E];
    const int64_t base = p.cell_base[E];
    if (n <= 0 || base < 0 || base + n > p.n_used) continue;
    const int c[3] = {cx - p.ncb + (t % p.nnt) * p.nt, cy - p.ncb + ((t / p.nnt) % p.nnt) * p.nt,
                      cz - p.ncb + (t / (p.nnt * p.nnt)) * p.nt};
    for (int l = lane; l < n; l += 32) {
      const int64_t ip = base + l;
      int i0[3];
      float w1[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double pos = ((double)c[d] + ((double)(uint16_t)p.xp[3 * ip + d] + 0.5) * (1.0 / 65536.0)) * scale - 0.5;
        const double f = floor(pos);
        i0[d] = (int)f;
        w1[d] = (float)(pos - f);  // weight of the upper point
      }
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int dx = k & 1, dy = (k >> 1) & 1, dz = k >> 2;
        const int gx = (i0[0] + dx + p.nw) % p.nw, gy = (i0[1] + dy + p.nw) % p.nw, gz = (i0[2] + dz + p.nw) % p.nw;
        const float w = (dx ? w1[0] : 1.f - w1[0]) * (dy ? w1[1] : 1.f - w1[1]) * (dz ? w1[2] : 1.f - w1[2]);
        atomicAdd(&p.grid[((int64_t)gz * p.nw + gy) * p.nw + gx], w);
      }
    }
  }
}

__global__ void k_density_contrast(float *grid, int64_t n, float scale) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) grid[i] = grid[i] * scale - 1.0f;
}

// one thread per mode of the half spectrum; block-local bins in shared memory
__global__ void __launch_bounds__(256) k_pk_bins(const cufftComplex *ck, int nw, int nbin, double *bins) {
  extern __shared__ double sb[];  // [4][nbin + 1]: modes, sum |k|, sum P, sum Delta^2
  for (int i = threadIdx.x; i < 4 * (nbin + 1); i += blockDim.x) sb[i] = 0.0;
  __syncthreads();
  const int nh = nw / 2 + 1, nyq = nw / 2;
  const int64_t nmodes = (int64_t)nw * nw * nh;
  const double norm = 1.0 / ((double)nw * nw * nw);
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nmodes; m += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(m % nh), j = (int)((m / nh) % nw), k = (int)(m / ((int64_t)nh * nw));
    if (i == 0 && j == 0 && k == 0) continue;
    if ((i == 0 || i == nyq) && j > nyq) continue;
    if ((i == 0 || i == nyq) && (j == 0 || j == nyq) && k > nyq) continue;
    const int kx = (i + nyq) % nw - nyq, ky = (j + nyq) % nw - nyq, kz = (k + nyq) % nw - nyq;
    const double kr = sqrt((double)kx * kx + (double)ky * ky + (double)kz * kz);
    const int b = (int)rint(kr);  // |k| is never a half-integer: rint = nint
    if (b > nbin) continue;
    const double pi = 3.14159265358979323846;
    double sinc = 1.0;
    const int kk[3] = {kx, ky, kz};
#pragma unroll
    for (int d = 0; d < 3; d++)
      if (kk[d] != 0) {
        const double a = pi * kk[d] / nw;
        sinc *= sin(a) / a;
      }
    const cufftComplex c = ck[m];
    const double re = c.x * norm, im = c.y * norm;
    const double s2 = sinc * sinc;
    const double pk = (re * re + im * im) / (s2 * s2);
    atomicAdd(&sb[b], 1.0);
    atomicAdd(&sb[(nbin + 1) + b], kr);
    atomicAdd(&sb[2 * (nbin + 1) + b], pk);
    atomicAdd(&sb[3 * (nbin + 1) + b], pk * 4.0 * pi * kr * kr * kr);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 4 * (nbin + 1); i += blockDim.x)
    if (sb[i] != 0.0) atomicAdd(&bins[i], sb[i]);
}

void launch_cic_grid(const Lay &L, int nw, const int32_t *rhoc, const int64_t *cell_base, const int16_t *xp,
                     int64_t n_used, float *grid, int num_sms, cudaStream_t s) {
  PowK p;
  p.n_used = n_used;
  p.nt = L.nt;
  p.ncb = L.ncb;
  p.nte = L.nte;
  p.nnt = L.nnt;
  p.nc = L.nc;
  p.nw = nw;
  p.ncells = (int64_t)L.ntile * L.nte * L.nte * L.nte;
  p.rhoc = rhoc;
  p.cell_base = cell_base;
  p.xp = xp;
  p.grid = grid;
  const int64_t blocks = (p.ncells + 7) / 8;
  k_cic_grid<<<(unsigned)std::min<int64_t>(blocks, (int64_t)num_sms * 32), 256, 0, s>>>(p);
}

void launch_density_contrast(float *grid, int64_t n, float scale, cudaStream_t s) {
  k_density_contrast<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(grid, n, scale);
}

size_t pk_bins_smem(int nbin) { return sizeof(double) * 4 * (nbin + 1); }

void launch_pk_bins(const cufftComplex *ck, int nw, int nbin, double *bins, int num_sms, cudaStream_t s) {
  const int64_t nmodes = (int64_t)nw * nw * (nw / 2 + 1);
  const int64_t blocks = (nmodes + 255) / 256;
  if (pk_bins_smem(nbin) > 48 * 1024)
    cudaFuncSetAttribute((const void *)k_pk_bins, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pk_bins_smem(nbin));
  k_pk_bins<<<(unsigned)std::min<int64_t>(blocks, (int64_t)num_sms * 8), 256, pk_bins_smem(nbin), s>>>(ck, nw, nbin,
                                                                                                      bins);
}

}  // namespace cube
