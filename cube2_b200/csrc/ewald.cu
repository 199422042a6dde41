// FP64 periodic direct summation of the softened force on sampled targets --
// the physics truth against which the kick's force errors are stated.  Not
// part of the kick.  Pair law F_ra(r, app) (basic_functions.f08:95-109),
// G = 1, unit masses, uniform neutralising background; the periodic 1/r^2
// sum is split the Ewald way:
//   real space : minimum image, r < rcut: (y-x)/r [erfc(a r)/r^2 + 2a/sqrt(pi) e^{-a^2 r^2}/r]
//   softening  : r < app: (y-x)/r (F_ra(r,app) - 1/r^2)
//   k space    : (4 pi/V) sum_{k!=0} k/k^2 e^{-k^2/4a^2} sin(k.(y-x)), half space doubled.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace cube {

__device__ double F_ra64(double r, double apm) {
  const double ep = 2 * r / apm;
  if (apm == 0 || ep > 2) return 1.0 / (r * r);
  const double e2 = ep * ep, e3 = e2 * ep, e4 = e3 * ep, e5 = e4 * ep, e6 = e5 * ep;
  if (ep > 1)
    return (1.0 / 35.0 / (apm * apm)) * (12 / e2 - 224 + 896 * ep - 840 * e2 + 224 * e3 + 70 * e4 - 48 * e5 + 7 * e6);
  if (ep > 0) return (1.0 / 35.0 / (apm * apm)) * (224 * ep - 224 * e3 + 70 * e4 + 48 * e5 - 21 * e6);
  return 0;
}

constexpr int kEwT = 128;

// grid.x: target blocks, grid.y: particle segments; partial forces added atomically
__global__ void __launch_bounds__(kEwT) k_ewald_real(const double *__restrict__ pos, int64_t n,
                                                     const int64_t *__restrict__ targets, int64_t nt, double L,
                                                     double app, double alpha, double rc2,
                                                     double *__restrict__ F) {
  __shared__ double sp[kEwT * 3];
  const int64_t t = (int64_t)blockIdx.x * kEwT + threadIdx.x;
  double x0 = 0, x1 = 0, x2 = 0;
  if (t < nt) {
    const int64_t it = targets[t];
    x0 = pos[3 * it];
    x1 = pos[3 * it + 1];
    x2 = pos[3 * it + 2];
  }
  const int64_t seg = (n + gridDim.y - 1) / gridDim.y;
  const int64_t j0 = (int64_t)blockIdx.y * seg, j1 = min(n, j0 + seg);
  const double c2 = 2.0 * alpha / sqrt(3.14159265358979323846);
  const double invL = 1.0 / L;
  double f0 = 0, f1 = 0, f2 = 0;
  for (int64_t jb = j0; jb < j1; jb += kEwT) {
    __syncthreads();
    const int64_t j = jb + threadIdx.x;
    if (j < j1) {
      sp[3 * threadIdx.x] = pos[3 * j];
      sp[3 * threadIdx.x + 1] = pos[3 * j + 1];
      sp[3 * threadIdx.x + 2] = pos[3 * j + 2];
    }
    __syncthreads();
    const int m = (int)min((int64_t)kEwT, j1 - jb);
    if (t < nt) {
      for (int q = 0; q < m; q++) {
        double d0 = sp[3 * q] - x0, d1 = sp[3 * q + 1] - x1, d2 = sp[3 * q + 2] - x2;
        d0 -= L * rint(d0 * invL);
        d1 -= L * rint(d1 * invL);
        d2 -= L * rint(d2 * invL);
        const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
        if (r2 == 0 || r2 >= rc2) continue;
        const double r = sqrt(r2);
        double s = erfc(alpha * r) / r2 + c2 * exp(-alpha * alpha * r2) / r;
        if (r < app) s += F_ra64(r, app) - 1.0 / r2;
        s /= r;
        f0 += s * d0;
        f1 += s * d1;
        f2 += s * d2;
      }
    }
  }
  if (t < nt) {
    atomicAdd(&F[3 * t], f0);
    atomicAdd(&F[3 * t + 1], f1);
    atomicAdd(&F[3 * t + 2], f2);
  }
}

// structure factor: grid.x over k-vector blocks, grid.y over particle segments
__global__ void __launch_bounds__(kEwT) k_ewald_sk(const double *__restrict__ pos, int64_t n,
                                                   const int *__restrict__ km, int nk, double w,
                                                   double *__restrict__ S) {
  __shared__ double sp[kEwT * 3];
  const int k = blockIdx.x * kEwT + threadIdx.x;
  double k0 = 0, k1 = 0, k2 = 0;
  if (k < nk) {
    k0 = w * km[3 * k];
    k1 = w * km[3 * k + 1];
    k2 = w * km[3 * k + 2];
  }
  const int64_t seg = (n + gridDim.y - 1) / gridDim.y;
  const int64_t j0 = (int64_t)blockIdx.y * seg, j1 = min(n, j0 + seg);
  double sc = 0, ss = 0;
  for (int64_t jb = j0; jb < j1; jb += kEwT) {
    __syncthreads();
    const int64_t j = jb + threadIdx.x;
    if (j < j1) {
      sp[3 * threadIdx.x] = pos[3 * j];
      sp[3 * threadIdx.x + 1] = pos[3 * j + 1];
      sp[3 * threadIdx.x + 2] = pos[3 * j + 2];
    }
    __syncthreads();
    const int m = (int)min((int64_t)kEwT, j1 - jb);
    if (k < nk)
      for (int q = 0; q < m; q++) {
        double s, c;
        sincos(k0 * sp[3 * q] + k1 * sp[3 * q + 1] + k2 * sp[3 * q + 2], &s, &c);
        sc += c;
        ss += s;
      }
  }
  if (k < nk) {
    atomicAdd(&S[2 * k], sc);
    atomicAdd(&S[2 * k + 1], ss);
  }
}

__global__ void k_ewald_kforce(const double *__restrict__ pos, const int64_t *__restrict__ targets, int64_t nt,
                               const int *__restrict__ km, int nk, const double *__restrict__ S, double w,
                               double alpha, double V, double *__restrict__ F) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int64_t it = targets[t];
  const double x0 = pos[3 * it], x1 = pos[3 * it + 1], x2 = pos[3 * it + 2];
  const double pi4 = 12.566370614359172953850573533118;
  double f0 = 0, f1 = 0, f2 = 0;
  for (int k = 0; k < nk; k++) {
    const double k0 = w * km[3 * k], k1 = w * km[3 * k + 1], k2 = w * km[3 * k + 2];
    const double kk = k0 * k0 + k1 * k1 + k2 * k2;
    double s, c;
    sincos(k0 * x0 + k1 * x1 + k2 * x2, &s, &c);
    const double sj = S[2 * k + 1] * c - S[2 * k] * s;
    const double g = 2.0 * (pi4 / V) * exp(-kk / (4 * alpha * alpha)) / kk * sj;
    f0 += g * k0;
    f1 += g * k1;
    f2 += g * k2;
  }
  F[3 * t] += f0;
  F[3 * t + 1] += f1;
  F[3 * t + 2] += f2;
}

int ewald_device(const double *pos, int64_t n, double box, double app, const int64_t *targets, int64_t nt,
                 double alpha, double rcut, int nmax, double *F) {
  std::vector<int> km;
  for (int mz = -nmax; mz <= nmax; mz++)
    for (int my = -nmax; my <= nmax; my++)
      for (int mx = -nmax; mx <= nmax; mx++) {
        if (mx * mx + my * my + mz * mz > nmax * nmax) continue;
        if (mz < 0 || (mz == 0 && my < 0) || (mz == 0 && my == 0 && mx <= 0)) continue;
        km.push_back(mx);
        km.push_back(my);
        km.push_back(mz);
      }
  const int nk = (int)(km.size() / 3);
  double *d_pos = nullptr, *d_F = nullptr, *d_S = nullptr;
  int64_t *d_t = nullptr;
  int *d_km = nullptr;
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t r) {
    if (r != cudaSuccess && e == cudaSuccess) e = r;
  };
  ck(cudaMalloc(&d_pos, sizeof(double) * 3 * n));
  ck(cudaMalloc(&d_F, sizeof(double) * 3 * nt));
  ck(cudaMalloc(&d_S, sizeof(double) * 2 * (nk > 0 ? nk : 1)));
  ck(cudaMalloc(&d_t, sizeof(int64_t) * (nt > 0 ? nt : 1)));
  ck(cudaMalloc(&d_km, sizeof(int) * 3 * (nk > 0 ? nk : 1)));
  if (e == cudaSuccess) {
    ck(cudaMemcpy(d_pos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    ck(cudaMemcpy(d_t, targets, sizeof(int64_t) * nt, cudaMemcpyHostToDevice));
    if (nk) ck(cudaMemcpy(d_km, km.data(), sizeof(int) * km.size(), cudaMemcpyHostToDevice));
    ck(cudaMemset(d_F, 0, sizeof(double) * 3 * nt));
    ck(cudaMemset(d_S, 0, sizeof(double) * 2 * (nk > 0 ? nk : 1)));
  }
  if (e == cudaSuccess && nt > 0) {
    const unsigned tb = (unsigned)((nt + kEwT - 1) / kEwT);
    unsigned segs = (unsigned)((148 * 16 + tb - 1) / tb);
    if ((int64_t)segs * 256 > n) segs = (unsigned)((n + 255) / 256);
    if (segs < 1) segs = 1;
    k_ewald_real<<<dim3(tb, segs), kEwT>>>(d_pos, n, d_t, nt, box, app, alpha, rcut * rcut, d_F);
    if (nk > 0) {
      const unsigned kb = (unsigned)((nk + kEwT - 1) / kEwT);
      unsigned ps = (unsigned)((148 * 16 + kb - 1) / kb);
      if ((int64_t)ps * 256 > n) ps = (unsigned)((n + 255) / 256);
      if (ps < 1) ps = 1;
      k_ewald_sk<<<dim3(kb, ps), kEwT>>>(d_pos, n, d_km, nk, 2 * 3.14159265358979323846 / box, d_S);
      k_ewald_kforce<<<(unsigned)((nt + 127) / 128), 128>>>(d_pos, d_t, nt, d_km, nk, d_S,
                                                           2 * 3.14159265358979323846 / box, alpha,
                                                           box * box * box, d_F);
    }
    ck(cudaGetLastError());
    ck(cudaMemcpy(F, d_F, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
  }
  cudaFree(d_pos);
  cudaFree(d_F);
  cudaFree(d_S);
  cudaFree(d_t);
  cudaFree(d_km);
  return e == cudaSuccess ? CUBE_OK : CUBE_ERR_CUDA;
}

}  // namespace cube
