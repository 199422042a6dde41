/*
 * ORACLE -- test infrastructure only.  CPU restatement of the reference PM3
 * fine-mesh force (the Fortran CPU path) and of its Green's-function
 * tabulation.  Only tests/, the smoke check and the CPU-baseline leg of the
 * benchmark load this; the product never does.
 *
 *   deposit  : kick.f90:418-468   (pm_thread, TSC weights :437-449, mass at :463)
 *   force    : kick.f90:545-568   (potential_to_force: phi/nwork^3 :552, 4-point
 *                                  weights parameters.f90:49-50)
 *   f2max    : kick.f90:494
 *   gather   : kick.f90:497-540   (TSC gather + kick dv*a_mid*dt/6/pi)
 *   Green    : Green/Green.f90:1-80 (Green_3D, FP64, alias sum n_int=2)
 *   PM1, PM2 : particle_mesh.f90 (pm_layer 1) and pm_thread with the PM2 parameters of
 *              kick.f90:82-88, the same deposit / force / gather on other meshes
 *
 * The FFT between deposit and force is done by the Python driver
 * (scipy.fft), the stand-in for FFTW/MKL which is not available here.
 *
 * Two mesh geometries are restated:
 *   mode 0 "subtile": the reference's per-subtile buffered mesh of side
 *          nft = nfp + 2*nfb (parameters.f90:62-65), deposit over the subtile
 *          plus nloop = 1 coarse cells, contributions outside the mesh dropped;
 *   mode 1 "periodic": one periodic mesh over the whole image of side
 *          n = ng * ratio_sf, deposit of every interior particle with periodic
 *          wrap (the same arithmetic with the buffer replaced by wrap-around).
 * Accumulation is in double (the reference accumulates in single); weights
 * and coordinates follow the reference's precision (l3, dx in real(4),
 * xpos in real(8), gridsize = real(4) 1/ratio_sf).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int ng, nnt, nns, ratio_cs, ngb;
} olay_t;

#define NC(L) ((L)->ng / (L)->ratio_cs)
#define NT(L) (NC(L) / (L)->nnt)
#define NTT(L) (NT(L) / (L)->nns)
#define NCB(L) ((L)->ngb / (L)->ratio_cs)
#define NTE(L) (NT(L) + 2 * NCB(L))

static inline int64_t rhoc_at(const olay_t *L, const int32_t *rhoc, int t, int k, int j, int i) {
  int64_t nte = NTE(L);
  return rhoc[(((int64_t)t * nte + k) * nte + j) * nte + i];
}

/* first storage index of the particles of extended cell (i,j,k) of tile t
 * (pp_force_kernel.c:203-209, kick.f90:289) */
static inline int64_t cell_base(const olay_t *L, const int32_t *rhoc, const int64_t *idx_b_r, int t,
                                int k, int j, int i) {
  int64_t nte = NTE(L);
  int64_t s = 0;
  for (int q = i; q < nte; q++) s += rhoc_at(L, rhoc, t, k, j, q);
  return idx_b_r[((int64_t)t * nte + k) * nte + j] - s;
}

/* kick.f90:292,437: (cell-1) + (int16(xp+ishift)+rshift)*x_resolution, exact in double */
static inline double decode(int c_minus_1, int16_t xp) {
  uint16_t u = (uint16_t)xp;
  return (double)c_minus_1 + ((double)u + 0.5) / 65536.0;
}

/* TSC weights, real(4) as in kick.f90:442-445 */
static inline void tsc_w(double xpos, int64_t *i0, float w[3]) {
  double f = floor(xpos);
  float l3 = (float)(xpos - f);
  *i0 = (int64_t)f;
  w[0] = (1.0f - l3) * (1.0f - l3) / 2.0f;
  w[2] = l3 * l3 / 2.0f;
  w[1] = 1.0f - w[0] - w[2];
}

static inline int64_t wrap(int64_t a, int64_t n) {
  a %= n;
  return a < 0 ? a + n : a;
}

/* mesh coordinate scale ratio_cs/gridsize with gridsize = real(4) 1/ratio_sf (kick.f90:157,438) */
static inline double mesh_scale(const olay_t *L, int rsf) {
  float gridsize = 1.0f / (float)rsf;
  return (double)L->ratio_cs / (double)gridsize;
}

/* ---------------- mode 1: periodic image mesh ---------------- */

/* Deposit every interior particle of every tile into rho[n][n][n] (unit mass).
 * Threads take whole z-planes of coarse cells; planes `stride` apart never touch
 * the same mesh points (the z-layer striping of kick.f90:425-429). */
static void deposit_periodic(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                             int64_t n, double sc, double *rho) {
  const int nnt = L->nnt, nt = NT(L), ncb = NCB(L), nc = NC(L);
  int stride = 3;
  while (nc % stride) stride++;
  memset(rho, 0, sizeof(double) * n * n * n);
  for (int phase = 0; phase < stride; phase++) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int gz = phase; gz < nc; gz += stride) {
      const int tz = gz / nt, k = gz % nt + ncb;
      for (int ty = 0; ty < nnt; ty++)
        for (int tx = 0; tx < nnt; tx++) {
          int t = (tz * nnt + ty) * nnt + tx;
          for (int j = ncb; j < ncb + nt; j++)
            for (int i = ncb; i < ncb + nt; i++) {
              int64_t np = rhoc_at(L, rhoc, t, k, j, i);
              int64_t base = cell_base(L, rhoc, idx_b_r, t, k, j, i);
              for (int64_t l = 0; l < np; l++) {
                const int16_t *q = xp + 3 * (base + l);
                double xs[3];
                xs[0] = decode(tx * nt + i - ncb, q[0]) * sc;
                xs[1] = decode(ty * nt + j - ncb, q[1]) * sc;
                xs[2] = decode(tz * nt + k - ncb, q[2]) * sc;
                int64_t c[3];
                float w[3][3];
                for (int d = 0; d < 3; d++) tsc_w(xs[d], &c[d], w[d]);
                for (int a = 0; a < 3; a++)
                  for (int b = 0; b < 3; b++)
                    for (int e = 0; e < 3; e++) {
                      int64_t X = wrap(c[0] + e - 1, n), Y = wrap(c[1] + b - 1, n), Z = wrap(c[2] + a - 1, n);
                      rho[(Z * n + Y) * n + X] += (double)(w[0][e] * w[1][b] * w[2][a]);
                    }
              }
            }
        }
    }
  }
}

void pm3o_deposit_periodic(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                           int rsf, double *rho) {
  deposit_periodic(L, xp, rhoc, idx_b_r, (int64_t)L->ng * rsf, mesh_scale(L, rsf), rho);
}

/* PM1 (particle_mesh.f90:18-60 with pm_layer 1): the periodic coarse mesh n = nc over the image,
 * mesh coordinate xpos * ratio_cs / gridsize with gridsize = real(ratio_cs), i.e. the global
 * coarse coordinate.  The reference deposits each tile with its nloop = 1 buffer cells and keeps
 * the tile's own mesh points, which places every physical particle's weights once, as here. */
void pm1o_deposit(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r, double *rho) {
  const float gs = (float)L->ratio_cs;
  deposit_periodic(L, xp, rhoc, idx_b_r, NC(L), (double)L->ratio_cs / (double)gs, rho);
}

/* potential_to_force on a periodic mesh: F_d(x) = sum_o w_o phi(x+o e_d) / n^3 * scale
 * (kick.f90:552-563), weights [(a-1)/4, -a/2, a/2, (1-a)/4], a = 4/3. */
void pm3o_force_periodic(int64_t n, const double *phi, double scale, double *force) {
  /* weight is a real(4) parameter built from alpha = 4./3 (parameters.f90:49-50) */
  const float alpha = 4.0f / 3.0f;
  const double wgt[4] = {(double)((alpha - 1) / 4), (double)(-alpha / 2), (double)(alpha / 2),
                         (double)((1 - alpha) / 4)};
  const int off[4] = {-2, -1, 1, 2};
  const double s = scale / ((double)n * (double)n * (double)n);
  const int64_t n3 = n * n * n;
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < n; z++)
    for (int64_t y = 0; y < n; y++)
      for (int64_t x = 0; x < n; x++) {
        double f[3] = {0, 0, 0};
        for (int o = 0; o < 4; o++) {
          f[0] += wgt[o] * phi[(z * n + y) * n + wrap(x + off[o], n)];
          f[1] += wgt[o] * phi[(z * n + wrap(y + off[o], n)) * n + x];
          f[2] += wgt[o] * phi[(wrap(z + off[o], n) * n + y) * n + x];
        }
        int64_t q = (z * n + y) * n + x;
        force[q] = f[0] * s;
        force[n3 + q] = f[1] * s;
        force[2 * n3 + q] = f[2] * s;
      }
}

/* f2max over all mesh points (kick.f90:494) */
double pm3o_f2max(int64_t npts, const double *force) {
  double m = 0;
  for (int64_t q = 0; q < npts; q++) {
    double v = force[q] * force[q] + force[npts + q] * force[npts + q] + force[2 * npts + q] * force[2 * npts + q];
    if (v > m) m = v;
  }
  return m;
}

/* Gather + kick for every interior particle (kick.f90:497-540):
 * dv = sum w F; vp[ip] += dv * kick; writes the applied dv (before kick) into acc[ip]
 * when acc != NULL; returns max |vp| per axis of the updated particles in vmax. */
static void gather_periodic(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                            int64_t n, double sc, const double *force, double kick, float *vp, double *acc,
                            float vmax[3]) {
  const int nnt = L->nnt, nt = NT(L), ncb = NCB(L);
  const int64_t n3 = n * n * n;
  float vm0 = 0, vm1 = 0, vm2 = 0;
  const int64_t ncell = (int64_t)nnt * nnt * nnt * nt * nt * nt;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : vm0, vm1, vm2)
  for (int64_t cidx = 0; cidx < ncell; cidx++) {
    int64_t r = cidx;
    const int i = (int)(r % nt) + ncb; r /= nt;
    const int j = (int)(r % nt) + ncb; r /= nt;
    const int k = (int)(r % nt) + ncb; r /= nt;
    const int t = (int)r;
    const int tx = t % nnt, ty = (t / nnt) % nnt, tz = t / (nnt * nnt);
    int64_t np = rhoc_at(L, rhoc, t, k, j, i);
    int64_t base = cell_base(L, rhoc, idx_b_r, t, k, j, i);
    for (int64_t l = 0; l < np; l++) {
      int64_t ip = base + l;
      const int16_t *q = xp + 3 * ip;
      double xs[3];
      xs[0] = decode(tx * nt + i - ncb, q[0]) * sc;
      xs[1] = decode(ty * nt + j - ncb, q[1]) * sc;
      xs[2] = decode(tz * nt + k - ncb, q[2]) * sc;
      int64_t c[3];
      float w[3][3];
      for (int d = 0; d < 3; d++) tsc_w(xs[d], &c[d], w[d]);
      double dv[3] = {0, 0, 0};
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          for (int e = 0; e < 3; e++) {
            int64_t X = wrap(c[0] + e - 1, n), Y = wrap(c[1] + b - 1, n), Z = wrap(c[2] + a - 1, n);
            int64_t m = (Z * n + Y) * n + X;
            double ww = (double)(w[0][e] * w[1][b] * w[2][a]);
            dv[0] += force[m] * ww;
            dv[1] += force[n3 + m] * ww;
            dv[2] += force[2 * n3 + m] * ww;
          }
      float av[3];
      for (int d = 0; d < 3; d++) {
        if (acc) acc[3 * ip + d] = dv[d];
        vp[3 * ip + d] = (float)((double)vp[3 * ip + d] + dv[d] * kick);
        av[d] = fabsf(vp[3 * ip + d]);
      }
      vm0 = av[0] > vm0 ? av[0] : vm0;
      vm1 = av[1] > vm1 ? av[1] : vm1;
      vm2 = av[2] > vm2 ? av[2] : vm2;
    }
  }
  vmax[0] = vm0;
  vmax[1] = vm1;
  vmax[2] = vm2;
}

void pm3o_gather_periodic(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                          int rsf, const double *force, double kick, float *vp, double *acc, float vmax[3]) {
  gather_periodic(L, xp, rhoc, idx_b_r, (int64_t)L->ng * rsf, mesh_scale(L, rsf), force, kick, vp, acc, vmax);
}

/* PM1 gather and kick (particle_mesh.f90:100-148) */
void pm1o_gather(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                 const double *force, double kick, float *vp, double *acc, float vmax[3]) {
  const float gs = (float)L->ratio_cs;
  gather_periodic(L, xp, rhoc, idx_b_r, NC(L), (double)L->ratio_cs / (double)gs, force, kick, vp, acc, vmax);
}

/* ---------------- PM2: per-tile buffered fine mesh (kick.f90:77-105, pm_thread :403-568) ---------------- */
/* Tile t (0-based), mesh side ngt = (nt + 2 ncb) ratio_cs, gridsize 1 (mesh coordinate = tile-local
 * fine coordinate), array index = Fortran index - (1 - ngb).  The deposit takes every stored cell
 * of the tile (nc1 - nloop .. nc2 + nloop with nloop = ncb), dropping weights outside the mesh;
 * the gather takes the physical cells. */
void pm2o_deposit(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r, int t,
                  double *rho) {
  const int ncb = NCB(L), nte = NTE(L);
  const int64_t nft = (int64_t)nte * L->ratio_cs, nfb = (int64_t)ncb * L->ratio_cs;
  const double sc = (double)L->ratio_cs / (double)1.0f;
  memset(rho, 0, sizeof(double) * nft * nft * nft);
  for (int k = 0; k < nte; k++)
    for (int j = 0; j < nte; j++)
      for (int i = 0; i < nte; i++) {
        int64_t np = rhoc_at(L, rhoc, t, k, j, i);
        int64_t base = cell_base(L, rhoc, idx_b_r, t, k, j, i);
        int cidx[3] = {i, j, k};
        for (int64_t l = 0; l < np; l++) {
          const int16_t *q = xp + 3 * (base + l);
          int64_t c[3];
          float w[3][3];
          for (int d = 0; d < 3; d++) tsc_w(decode(cidx[d] - ncb, q[d]) * sc, &c[d], w[d]);
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              for (int e = 0; e < 3; e++) {
                int64_t X = c[0] + e - 1 + nfb, Y = c[1] + b - 1 + nfb, Z = c[2] + a - 1 + nfb;
                if (X < 0 || X >= nft || Y < 0 || Y >= nft || Z < 0 || Z >= nft) continue;
                rho[(Z * nft + Y) * nft + X] += (double)(w[0][e] * w[1][b] * w[2][a]);
              }
        }
      }
}

void pm2o_gather(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r, int t,
                 const double *force, double kick, float *vp, double *acc, float vmax[3]) {
  const int ncb = NCB(L), nt = NT(L), nte = NTE(L);
  const int64_t nft = (int64_t)nte * L->ratio_cs, nfb = (int64_t)ncb * L->ratio_cs, n3 = nft * nft * nft;
  const double sc = (double)L->ratio_cs / (double)1.0f;
  for (int k = ncb; k < ncb + nt; k++)
    for (int j = ncb; j < ncb + nt; j++)
      for (int i = ncb; i < ncb + nt; i++) {
        int64_t np = rhoc_at(L, rhoc, t, k, j, i);
        int64_t base = cell_base(L, rhoc, idx_b_r, t, k, j, i);
        int cidx[3] = {i, j, k};
        for (int64_t l = 0; l < np; l++) {
          int64_t ip = base + l;
          const int16_t *q = xp + 3 * ip;
          int64_t c[3];
          float w[3][3];
          for (int d = 0; d < 3; d++) tsc_w(decode(cidx[d] - ncb, q[d]) * sc, &c[d], w[d]);
          double dv[3] = {0, 0, 0};
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              for (int e = 0; e < 3; e++) {
                int64_t m = ((c[2] + a - 1 + nfb) * nft + (c[1] + b - 1 + nfb)) * nft + (c[0] + e - 1 + nfb);
                double ww = (double)(w[0][e] * w[1][b] * w[2][a]);
                dv[0] += force[m] * ww;
                dv[1] += force[n3 + m] * ww;
                dv[2] += force[2 * n3 + m] * ww;
              }
          for (int d = 0; d < 3; d++) {
            if (acc) acc[3 * ip + d] = dv[d];
            vp[3 * ip + d] = (float)((double)vp[3 * ip + d] + dv[d] * kick);
            float av = fabsf(vp[3 * ip + d]);
            if (av > vmax[d]) vmax[d] = av;
          }
        }
      }
}

/* ---------------- mode 0: per-subtile buffered mesh ---------------- */
/* Subtile `it` (0-based, ordering of initialize.f90:207-224): rows of ixyz3 are
 * [sx,sy,sz,tx,ty,tz] 1-based.  Mesh side nft = nfp + 2 nfb with
 * nfp = ntt*ratio_cs*rsf and nfb = ratio_cs*rsf (parameters.f90:62-65).  Mesh
 * array index m = Fortran index - (1 - nfb). */

void pm3o_deposit_subtile(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                          const int32_t *ixyz3, int it, int rsf, double *rho) {
  const int nnt = L->nnt, ncb = NCB(L), ntt = NTT(L);
  const int sx = ixyz3[6 * it + 0] - 1, sy = ixyz3[6 * it + 1] - 1, sz = ixyz3[6 * it + 2] - 1;
  const int tx = ixyz3[6 * it + 3] - 1, ty = ixyz3[6 * it + 4] - 1, tz = ixyz3[6 * it + 5] - 1;
  const int t = (tz * nnt + ty) * nnt + tx;
  const int64_t nfp = (int64_t)ntt * L->ratio_cs * rsf, nfb = (int64_t)L->ratio_cs * rsf, nft = nfp + 2 * nfb;
  const double sc = mesh_scale(L, rsf);
  const int us[3] = {sx, sy, sz};
  memset(rho, 0, sizeof(double) * nft * nft * nft);
  /* Fortran cells nc1-nloop .. nc2+nloop (kick.f90:429-432), C index = Fortran + ncb - 1 */
  int lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = us[d] * ntt + ncb - 1;
    hi[d] = (us[d] + 1) * ntt + ncb;
  }
  for (int k = lo[2]; k <= hi[2]; k++)
    for (int j = lo[1]; j <= hi[1]; j++)
      for (int i = lo[0]; i <= hi[0]; i++) {
        int64_t np = rhoc_at(L, rhoc, t, k, j, i);
        int64_t base = cell_base(L, rhoc, idx_b_r, t, k, j, i);
        int cidx[3] = {i, j, k};
        for (int64_t l = 0; l < np; l++) {
          const int16_t *q = xp + 3 * (base + l);
          int64_t c[3];
          float w[3][3];
          for (int d = 0; d < 3; d++) {
            double xpos = decode(cidx[d] - ncb, q[d]) * sc - (double)us[d] * (double)nfp;
            tsc_w(xpos, &c[d], w[d]);
          }
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              for (int e = 0; e < 3; e++) {
                int64_t X = c[0] + e - 1 + nfb, Y = c[1] + b - 1 + nfb, Z = c[2] + a - 1 + nfb;
                if (X < 0 || X >= nft || Y < 0 || Y >= nft || Z < 0 || Z >= nft) continue;
                rho[(Z * nft + Y) * nft + X] += (double)(w[0][e] * w[1][b] * w[2][a]);
              }
        }
      }
}

/* f2max over the physical force points, Fortran 1..nfp -> array nfb..nfb+nfp-1 (kick.f90:494) */
double pm3o_f2max_subtile(int64_t nft, int64_t nfp, int64_t nfb, const double *force) {
  const int64_t n3 = nft * nft * nft;
  double m = 0;
  for (int64_t z = nfb; z < nfb + nfp; z++)
    for (int64_t y = nfb; y < nfb + nfp; y++)
      for (int64_t x = nfb; x < nfb + nfp; x++) {
        int64_t q = (z * nft + y) * nft + x;
        double v = force[q] * force[q] + force[n3 + q] * force[n3 + q] + force[2 * n3 + q] * force[2 * n3 + q];
        if (v > m) m = v;
      }
  return m;
}

/* gather + kick for the subtile's own particles (kick.f90:503-536) */
void pm3o_gather_subtile(const olay_t *L, const int16_t *xp, const int32_t *rhoc, const int64_t *idx_b_r,
                         const int32_t *ixyz3, int it, int rsf, const double *force, double kick, float *vp,
                         double *acc, float vmax[3]) {
  const int nnt = L->nnt, ncb = NCB(L), ntt = NTT(L);
  const int sx = ixyz3[6 * it + 0] - 1, sy = ixyz3[6 * it + 1] - 1, sz = ixyz3[6 * it + 2] - 1;
  const int tx = ixyz3[6 * it + 3] - 1, ty = ixyz3[6 * it + 4] - 1, tz = ixyz3[6 * it + 5] - 1;
  const int t = (tz * nnt + ty) * nnt + tx;
  const int64_t nfp = (int64_t)ntt * L->ratio_cs * rsf, nfb = (int64_t)L->ratio_cs * rsf, nft = nfp + 2 * nfb;
  const int64_t n3 = nft * nft * nft;
  const double sc = mesh_scale(L, rsf);
  const int us[3] = {sx, sy, sz};
  for (int k = us[2] * ntt + ncb; k < (us[2] + 1) * ntt + ncb; k++)
    for (int j = us[1] * ntt + ncb; j < (us[1] + 1) * ntt + ncb; j++)
      for (int i = us[0] * ntt + ncb; i < (us[0] + 1) * ntt + ncb; i++) {
        int64_t np = rhoc_at(L, rhoc, t, k, j, i);
        int64_t base = cell_base(L, rhoc, idx_b_r, t, k, j, i);
        int cidx[3] = {i, j, k};
        for (int64_t l = 0; l < np; l++) {
          int64_t ip = base + l;
          const int16_t *q = xp + 3 * ip;
          int64_t c[3];
          float w[3][3];
          for (int d = 0; d < 3; d++) {
            double xpos = decode(cidx[d] - ncb, q[d]) * sc - (double)us[d] * (double)nfp;
            tsc_w(xpos, &c[d], w[d]);
          }
          double dv[3] = {0, 0, 0};
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              for (int e = 0; e < 3; e++) {
                int64_t m = ((c[2] + a - 1 + nfb) * nft + (c[1] + b - 1 + nfb)) * nft + (c[0] + e - 1 + nfb);
                double ww = (double)(w[0][e] * w[1][b] * w[2][a]);
                dv[0] += force[m] * ww;
                dv[1] += force[n3 + m] * ww;
                dv[2] += force[2 * n3 + m] * ww;
              }
          for (int d = 0; d < 3; d++) {
            if (acc) acc[3 * ip + d] = dv[d];
            vp[3 * ip + d] = (float)((double)vp[3 * ip + d] + dv[d] * kick);
            float av = fabsf(vp[3 * ip + d]);
            if (av > vmax[d]) vmax[d] = av;
          }
        }
      }
}

/* ---------------- Green's function (Green/Green.f90:1-80, kshift = 0) ---------------- */
/* Gk(k1,k2,k3) for k1 in 1..n/2+1, k2,k3 in 1..n, stored C-order [k3][k2][k1]; p_order = p (1 CIC, 2 TSC). */
void pm3o_green(int64_t n, double apm_soft, double apm_range, double gridsize, int p_order, float *G) {
  /* Fortran literals 4./3, 2./15 and 1./nglobal are default (single) reals and
   * gridsize is real(4); they are rounded the same way here. */
  const double pi = 4.0 * atan(1.0);
  const double alpha = (double)(4.0f / 3.0f);
  const double c215 = (double)(2.0f / 15.0f);
  const int n_int = 2;
  const int64_t n1 = n / 2 + 1;
  double *fs = (double *)malloc(sizeof(double) * n);
  const double inv_n = (double)(1.0f / (float)n);
  for (int64_t k = 1; k <= n; k++) {
    int64_t m = (k + n / 2 - 1) % n - n / 2;
    fs[k - 1] = 2.0 * pi * inv_n * (double)m;
  }
  const float gs = (float)gridsize;
  const double gpow = (double)(gs * gs);
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int64_t k3 = 0; k3 < n; k3++)
    for (int64_t k2 = 0; k2 < n; k2++)
      for (int64_t k1 = 0; k1 < n1; k1++) {
        double kv[3] = {fs[k1], fs[k2], fs[k3]};
        double D[3], ur[3] = {0, 0, 0}, u2n = 1;
        for (int d = 0; d < 3; d++) {
          D[d] = alpha * sin(kv[d]) + (1 - alpha) * sin(2 * kv[d]) / 2;
          double s = sin(kv[d] / 2);
          u2n *= 1 - s * s + c215 * s * s * s * s;
        }
        for (int i3 = -n_int; i3 <= n_int; i3++)
          for (int i2 = -n_int; i2 <= n_int; i2++)
            for (int i1 = -n_int; i1 <= n_int; i1++) {
              double kn[3] = {kv[0] + 2 * pi * i1, kv[1] + 2 * pi * i2, kv[2] + 2 * pi * i3};
              double kmag = sqrt(kn[0] * kn[0] + kn[1] * kn[1] + kn[2] * kn[2]);
              double U = 1;
              for (int d = 0; d < 3; d++) U *= (kn[d] == 0) ? 1.0 : sin(kn[d] / 2) / (kn[d] / 2);
              U = pow(U, 2 * p_order + 2);
              double y = apm_soft * kmag / 2, Ss, Sr;
              Ss = (kmag == 0) ? 1.0 : 12 * pow(y, -4) * (2 - 2 * cos(y) - y * sin(y));
              if (apm_range == 0)
                Sr = 0;
              else if (kmag == 0)
                Sr = 1;
              else {
                double yr = apm_range * kmag / 2;
                Sr = 12 * pow(yr, -4) * (2 - 2 * cos(yr) - yr * sin(yr));
              }
              double f = (Ss * Ss - Sr * Sr) / (kmag * kmag);
              for (int d = 0; d < 3; d++) ur[d] += U * kn[d] * f;
            }
        double num = D[0] * ur[0] + D[1] * ur[1] + D[2] * ur[2];
        double den = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
        G[(k3 * n + k2) * n1 + k1] = (float)(4 * pi * num / den / (u2n * u2n) / gpow);
      }
  /* Gk(::n/2, ::n/2, ::n/2) = 0 (Green.f90:71): the 8 corners {0, n/2}^3 */
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) G[((a * (n / 2)) * n + b * (n / 2)) * n1 + c * (n / 2)] = 0.0f;
  free(fs);
}

/* The same table from a quarter of the work: the wavenumbers of indices k and n - k along the
 * second and third axes are m and -m, and Green_3D is even in each component, so rows k2, k3 in
 * (n/2, n) are copies of rows n - k2, n - k3.  The alias sums of a mirrored row run in the
 * opposite order, so the copies can differ from pm3o_green in the last bit of the FP64 sum (far
 * below the float rounding of the result).  Used where a large table is tabulated on the host
 * outside a timed region. */
void pm3o_green_mirrored(int64_t n, double apm_soft, double apm_range, double gridsize, int p_order, float *G) {
  const int64_t n1 = n / 2 + 1, h = n / 2;
  const int64_t m = h + 1; /* rows 0 .. n/2 of each mirrored axis */
  float *Q = (float *)malloc(sizeof(float) * (size_t)(m * m * n1));
  /* tabulate the rows k2, k3 in 0..n/2 on an n-periodic grid: pm3o_green's loop restricted */
  const double pi = 4.0 * atan(1.0);
  const double alpha = (double)(4.0f / 3.0f);
  const double c215 = (double)(2.0f / 15.0f);
  const int n_int = 2;
  double *fs = (double *)malloc(sizeof(double) * n);
  const double inv_n = (double)(1.0f / (float)n);
  for (int64_t k = 1; k <= n; k++) {
    int64_t mm = (k + n / 2 - 1) % n - n / 2;
    fs[k - 1] = 2.0 * pi * inv_n * (double)mm;
  }
  const float gs = (float)gridsize;
  const double gpow = (double)(gs * gs);
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int64_t k3 = 0; k3 < m; k3++)
    for (int64_t k2 = 0; k2 < m; k2++)
      for (int64_t k1 = 0; k1 < n1; k1++) {
        double kv[3] = {fs[k1], fs[k2], fs[k3]};
        double D[3], ur[3] = {0, 0, 0}, u2n = 1;
        for (int d = 0; d < 3; d++) {
          D[d] = alpha * sin(kv[d]) + (1 - alpha) * sin(2 * kv[d]) / 2;
          double s = sin(kv[d] / 2);
          u2n *= 1 - s * s + c215 * s * s * s * s;
        }
        for (int i3 = -n_int; i3 <= n_int; i3++)
          for (int i2 = -n_int; i2 <= n_int; i2++)
            for (int i1 = -n_int; i1 <= n_int; i1++) {
              double kn[3] = {kv[0] + 2 * pi * i1, kv[1] + 2 * pi * i2, kv[2] + 2 * pi * i3};
              double kmag = sqrt(kn[0] * kn[0] + kn[1] * kn[1] + kn[2] * kn[2]);
              double U = 1;
              for (int d = 0; d < 3; d++) U *= (kn[d] == 0) ? 1.0 : sin(kn[d] / 2) / (kn[d] / 2);
              U = pow(U, 2 * p_order + 2);
              double y = apm_soft * kmag / 2, Ss, Sr;
              Ss = (kmag == 0) ? 1.0 : 12 * pow(y, -4) * (2 - 2 * cos(y) - y * sin(y));
              if (apm_range == 0)
                Sr = 0;
              else if (kmag == 0)
                Sr = 1;
              else {
                double yr = apm_range * kmag / 2;
                Sr = 12 * pow(yr, -4) * (2 - 2 * cos(yr) - yr * sin(yr));
              }
              double f = (Ss * Ss - Sr * Sr) / (kmag * kmag);
              for (int d = 0; d < 3; d++) ur[d] += U * kn[d] * f;
            }
        double num = D[0] * ur[0] + D[1] * ur[1] + D[2] * ur[2];
        double den = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
        Q[(k3 * m + k2) * n1 + k1] = (float)(4 * pi * num / den / (u2n * u2n) / gpow);
      }
#pragma omp parallel for collapse(2)
  for (int64_t k3 = 0; k3 < n; k3++)
    for (int64_t k2 = 0; k2 < n; k2++) {
      const int64_t q3 = k3 <= h ? k3 : n - k3, q2 = k2 <= h ? k2 : n - k2;
      memcpy(G + (k3 * n + k2) * n1, Q + (q3 * m + q2) * n1, sizeof(float) * (size_t)n1);
    }
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) G[((a * (n / 2)) * n + b * (n / 2)) * n1 + c * (n / 2)] = 0.0f;
  free(fs);
  free(Q);
}
