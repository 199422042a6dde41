// PM3 fine-mesh force (kick.f90:403-568, pm3_fft_cuda.cu:276-391).
//
// Pipeline per batch of meshes:
//   deposit  TSC weights of every particle of the job's coarse cells into the
//            mesh (kick.f90:420-468); one warp per coarse cell, float atomics
//            (the cost follows the particles, not the mesh, which matters for
//            clustered boxes where most mesh bricks are nearly empty);
//   R2C      cuFFT;
//   k-space  one kernel multiplies by the Green table and by the spectral
//            symbol of the 4-point difference, i*D(k) with
//            D = a sin k + (1-a) sin 2k / 2, a = 4/3 -- the exact Fourier image
//            of potential_to_force (kick.f90:545-568) on the FFT mesh -- and
//            writes the three force spectra;
//   C2R      cuFFT, batched over the 3 components (three separate arrays: a
//            stride-4 interleaved output measured slower for both cuFFT and
//            the gather);
//   f2max    max |F|^2 over the physical mesh points (kick.f90:494), float4
//            loads along x;
//   gather   TSC gather of the force at each active particle and the kick
//            vp += dv * a_mid*dt/(6 pi) (kick.f90:497-540).
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
  float *rho;
  const cufftComplex *rhok;
  cufftComplex *fk;
  const float *force;  // [slot][3][n^3]
  const float *green;
  const float *dtab;
  float gscale;  // mass / n^3
  float kick;
  float *vp;
  float *out;
  int want_vmax;
  int fphys_lo, fphys_n;
  int nslots;
};

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
#pragma unroll
    for (int c = 0; c < 3; c++) {
      int64_t Z = iz + c - 1;
      if (p.wrap) Z = wrapi(Z, n); else if (Z < 0 || Z >= n) continue;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        int64_t Y = iy + b - 1;
        if (p.wrap) Y = wrapi(Y, n); else if (Y < 0 || Y >= n) continue;
#pragma unroll
        for (int a = 0; a < 3; a++) {
          int64_t X = ix + a - 1;
          if (p.wrap) X = wrapi(X, n); else if (X < 0 || X >= n) continue;
          atomicAdd(R + (Z * n + Y) * n + X, (wx[a] * wy[b]) * wz[c]);
        }
      }
    }
  }
}

// fk[slot][d] = i * D_d(k) * G(k) * mass / n^3 * rhok[slot]
__global__ void k_kspace(PM3K p) {
  const int64_t total = p.nk * p.nslots;
  const int n = p.n, nh = n / 2 + 1;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int slot = (int)(e / p.nk);
    const int64_t k = e - (int64_t)slot * p.nk;
    const int kx = (int)(k % nh);
    const int ky = (int)((k / nh) % n);
    const int kz = (int)(k / ((int64_t)nh * n));
    const float g = p.green[k] * p.gscale;
    const cufftComplex c = p.rhok[e];
    const float re = c.x * g, im = c.y * g;
    const float D[3] = {p.dtab[kx], p.dtab[ky], p.dtab[kz]};
    cufftComplex *F = p.fk + (int64_t)slot * 3 * p.nk + k;
#pragma unroll
    for (int d = 0; d < 3; d++) F[d * p.nk] = make_float2(-D[d] * im, D[d] * re);
  }
}

__global__ void k_f2max(PM3K p) {
  float m = 0.f;
  const int64_t nph = (int64_t)p.fphys_n * p.fphys_n * p.fphys_n;
  const int64_t total = nph * p.nslots;
  const int64_t n = p.n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int slot = (int)(e / nph);
    const int64_t r = e - slot * nph;
    const int64_t x = r % p.fphys_n + p.fphys_lo, y = (r / p.fphys_n) % p.fphys_n + p.fphys_lo,
                  z = r / ((int64_t)p.fphys_n * p.fphys_n) + p.fphys_lo;
    const int64_t q = (z * n + y) * n + x;
    const float *F = p.force + (int64_t)slot * 3 * p.n3;
    const float a = F[q], b = F[p.n3 + q], c = F[2 * p.n3 + q];
    m = fmaxf(m, a * a + b * b + c * c);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&p.out[0], m);
}

// f2max with float4 loads along x (the physical region starts and ends on multiples of 4)
__global__ void k_f2max_v4(PM3K p) {
  float m = 0.f;
  const int64_t g4 = p.fphys_n / 4;
  const int64_t nph = g4 * p.fphys_n * p.fphys_n;
  const int64_t total = nph * p.nslots;
  const int64_t n = p.n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int slot = (int)(e / nph);
    const int64_t r = e - slot * nph;
    const int64_t x = 4 * (r % g4) + p.fphys_lo, y = (r / g4) % p.fphys_n + p.fphys_lo,
                  z = r / (g4 * p.fphys_n) + p.fphys_lo;
    const int64_t q = (z * n + y) * n + x;
    const float *F = p.force + (int64_t)slot * 3 * p.n3;
    const float4 a = __ldg(reinterpret_cast<const float4 *>(F + q));
    const float4 b = __ldg(reinterpret_cast<const float4 *>(F + p.n3 + q));
    const float4 c = __ldg(reinterpret_cast<const float4 *>(F + 2 * p.n3 + q));
    m = fmaxf(m, fmaxf(fmaxf(a.x * a.x + b.x * b.x + c.x * c.x, a.y * a.y + b.y * b.y + c.y * c.y),
                       fmaxf(a.z * a.z + b.z * b.z + c.z * c.z, a.w * a.w + b.w * b.w + c.w * c.w)));
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&p.out[0], m);
}

__global__ void __launch_bounds__(kWarps * 32) k_gather(PM3K p) {
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
        const int64_t Z = p.wrap ? wrapi(iz + c - 1, n) : iz + c - 1;
#pragma unroll
        for (int b = 0; b < 3; b++) {
          const int64_t Y = p.wrap ? wrapi(iy + b - 1, n) : iy + b - 1;
#pragma unroll
          for (int a = 0; a < 3; a++) {
            const int64_t X = p.wrap ? wrapi(ix + a - 1, n) : ix + a - 1;
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
  p.fk = a.fk;
  p.force = a.force;
  p.green = a.green;
  p.dtab = a.dtab;
  p.gscale = (float)((double)a.mass / ((double)a.n * a.n * a.n));
  p.kick = a.kick;
  p.vp = a.vp;
  p.out = a.out;
  p.want_vmax = a.want_vmax;
  p.fphys_lo = a.fphys_lo;
  p.fphys_n = a.fphys_n;
  p.nslots = a.nslots;
  return p;
}

void launch_pm3_deposit(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  const int64_t warps = (int64_t)a.rdep[0] * a.rdep[1] * a.rdep[2] * a.njobs;
  k_deposit<<<(unsigned)((warps + kWarps - 1) / kWarps), kWarps * 32, 0, s>>>(p);
}

void launch_pm3_kspace(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  k_kspace<<<148 * 8, 256, 0, s>>>(p);
}

void launch_pm3_f2max(const PM3Args &a, cudaStream_t s) {
  PM3K p = make_k(a);
  if (a.fphys_lo % 4 == 0 && a.fphys_n % 4 == 0 && a.n % 4 == 0)
    k_f2max_v4<<<148 * 8, 256, 0, s>>>(p);
  else
    k_f2max<<<148 * 8, 256, 0, s>>>(p);
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
