/*
 * ORACLE -- test infrastructure only.  FP64 periodic direct summation of the
 * softened gravitational force (the physics truth against which force errors
 * are stated).  Not used by the product path.
 *
 * Pair law: F_ra(r, app) of basic_functions.f08:95-109 (S2 / uniform-sphere
 * softening; equals 1/r^2 for r > app), G = 1, unit masses, periodic box of
 * side L with a uniform neutralising background (the k = 0 mode removed, as
 * in the mesh solver).  The periodic 1/r^2 sum is split the Ewald way:
 *   real space : (y-x)/r * [erfc(a r)/r^2 + 2a/sqrt(pi) exp(-a^2 r^2)/r], minimum image, r < rcut
 *   k space    : (4 pi / V) sum_{k != 0} k/k^2 exp(-k^2/4a^2) sin(k.(y-x))
 *   softening  : (y-x)/r * (F_ra(r,app) - 1/r^2) for r < app
 * rcut <= L/2 keeps the minimum image exact; choose a so that erfc(a rcut)
 * and exp(-kmax^2/4a^2) are below the accuracy wanted.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* basic_functions.f08:95-109 in double */
static double F_ra64(double r, double apm) {
  double ep = 2 * r / apm;
  if (apm == 0 || ep > 2) return 1.0 / (r * r);
  if (ep > 1)
    return (1.0 / 35.0 / (apm * apm)) *
           (12 / (ep * ep) - 224 + 896 * ep - 840 * ep * ep + 224 * pow(ep, 3) + 70 * pow(ep, 4) -
            48 * pow(ep, 5) + 7 * pow(ep, 6));
  if (ep > 0)
    return (1.0 / 35.0 / (apm * apm)) *
           (224 * ep - 224 * pow(ep, 3) + 70 * pow(ep, 4) + 48 * pow(ep, 5) - 21 * pow(ep, 6));
  return 0;
}

double cube_oracle_F_ra64(double r, double apm) { return F_ra64(r, apm); }

/* Forces on the Nt target particles (indices into pos) from all N particles. */
void ewald_forces(int64_t N, const double *pos, double L, double app, int64_t Nt, const int64_t *targets,
                  double alpha, double rcut, int nmax, double *F) {
  const double rc2 = rcut * rcut;
  const double c2 = 2.0 * alpha / sqrt(M_PI);
  /* real space + softening */
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t t = 0; t < Nt; t++) {
    const double *x = pos + 3 * targets[t];
    double f[3] = {0, 0, 0};
    for (int64_t j = 0; j < N; j++) {
      double d[3];
      for (int q = 0; q < 3; q++) {
        d[q] = pos[3 * j + q] - x[q];
        d[q] -= L * nearbyint(d[q] / L);
      }
      double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 == 0 || r2 >= rc2) continue;
      double r = sqrt(r2);
      double s = erfc(alpha * r) / r2 + c2 * exp(-alpha * alpha * r2) / r;
      if (r < app) s += F_ra64(r, app) - 1.0 / r2;
      s /= r;
      f[0] += s * d[0];
      f[1] += s * d[1];
      f[2] += s * d[2];
    }
    F[3 * t + 0] = f[0];
    F[3 * t + 1] = f[1];
    F[3 * t + 2] = f[2];
  }
  /* k space: half space of integer vectors m with |m| <= nmax, k = 2 pi m / L */
  const int nm = 2 * nmax + 1;
  int64_t nk = 0;
  int *km = (int *)malloc(sizeof(int) * 3 * nm * nm * nm);
  for (int mz = -nmax; mz <= nmax; mz++)
    for (int my = -nmax; my <= nmax; my++)
      for (int mx = -nmax; mx <= nmax; mx++) {
        if (mx * mx + my * my + mz * mz > nmax * nmax) continue;
        /* half space: first nonzero component positive */
        if (mz < 0 || (mz == 0 && my < 0) || (mz == 0 && my == 0 && mx <= 0)) continue;
        km[3 * nk] = mx;
        km[3 * nk + 1] = my;
        km[3 * nk + 2] = mz;
        nk++;
      }
  double *Sc = (double *)calloc(nk, sizeof(double));
  double *Ss = (double *)calloc(nk, sizeof(double));
  const double w = 2 * M_PI / L;
#pragma omp parallel
  {
    double *lc = (double *)calloc(nk, sizeof(double));
    double *ls = (double *)calloc(nk, sizeof(double));
    double *ex = (double *)malloc(sizeof(double) * 2 * 3 * nm);
#pragma omp for schedule(static)
    for (int64_t j = 0; j < N; j++) {
      for (int q = 0; q < 3; q++)
        for (int m = -nmax; m <= nmax; m++) {
          double a = w * m * pos[3 * j + q];
          ex[2 * (q * nm + m + nmax)] = cos(a);
          ex[2 * (q * nm + m + nmax) + 1] = sin(a);
        }
      for (int64_t k = 0; k < nk; k++) {
        const double *a = ex + 2 * (0 * nm + km[3 * k] + nmax);
        const double *b = ex + 2 * (1 * nm + km[3 * k + 1] + nmax);
        const double *c = ex + 2 * (2 * nm + km[3 * k + 2] + nmax);
        double re = a[0] * b[0] - a[1] * b[1], im = a[0] * b[1] + a[1] * b[0];
        double re2 = re * c[0] - im * c[1], im2 = re * c[1] + im * c[0];
        lc[k] += re2;
        ls[k] += im2;
      }
    }
#pragma omp critical
    for (int64_t k = 0; k < nk; k++) {
      Sc[k] += lc[k];
      Ss[k] += ls[k];
    }
    free(lc);
    free(ls);
    free(ex);
  }
  const double V = L * L * L;
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < Nt; t++) {
    const double *x = pos + 3 * targets[t];
    double f[3] = {0, 0, 0};
    for (int64_t k = 0; k < nk; k++) {
      double kv[3] = {w * km[3 * k], w * km[3 * k + 1], w * km[3 * k + 2]};
      double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      double kx = kv[0] * x[0] + kv[1] * x[1] + kv[2] * x[2];
      /* sum_j sin(k.(y_j - x)) = Ss cos(k.x) - Sc sin(k.x) */
      double sj = Ss[k] * cos(kx) - Sc[k] * sin(kx);
      double g = 2.0 * (4 * M_PI / V) * exp(-k2 / (4 * alpha * alpha)) / k2 * sj;
      f[0] += g * kv[0];
      f[1] += g * kv[1];
      f[2] += g * kv[2];
    }
    F[3 * t + 0] += f[0];
    F[3 * t + 1] += f[1];
    F[3 * t + 2] += f[2];
  }
  free(km);
  free(Sc);
  free(Ss);
}
