// Checkpoint files of one image (checkpoint.f90:11-38, read back by
// particle_initialization.f90:19-60): Fortran stream files without record markers,
//   <prefix>info<suffix>  the sim_header of parameters.f90:141-164: 13 int64 then 19 real(4)
//   <prefix>xp<suffix>    int16 [nplocal][3]  physical particles in storage order
//   <prefix>vp<suffix>    real(4) [nplocal][3]
//   <prefix>np<suffix>    int32 rhoc(1:nt,1:nt,1:nt,:,:,:), C view [nnt^3 tiles][nt][nt][nt]
//   <prefix>id<suffix>    int64 [nplocal] particle ids (PID builds)
// The reference writes them right after a drift, when the image holds its physical particles
// only, tile by tile and row by row (drift.f90:121-133); the writer here takes an image with
// buffers and writes its physical particles in that same order.  Host code only.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace cube {

static_assert(sizeof(cube_sim_header) >= kSimHeaderBytes, "header struct");

static void header_to_bytes(const cube_sim_header &h, unsigned char *b) {
  const int64_t ints[13] = {h.nplocal, h.npglobal, h.izipx,    h.izipv,         h.image,
                            h.nn,      h.nnt,      h.nt,       h.ncell,         h.ncb,
                            h.timestep, h.cur_checkpoint, h.cur_halofind};
  const float reals[19] = {h.a,          h.t,   h.tau, h.dt_pp,   h.dt_pm3,  h.dt_pm2,    h.dt_pm1,
                           h.dt_vmax,    h.mass_p_cdm, h.box,     h.h0,      h.omega_m,   h.omega_l,
                           h.s8,         h.vsim2phys,  h.sigma_vres, h.sigma_vi, h.z_i, h.vz_max};
  std::memcpy(b, ints, sizeof(ints));
  std::memcpy(b + sizeof(ints), reals, sizeof(reals));
}

static void header_from_bytes(const unsigned char *b, cube_sim_header &h) {
  int64_t ints[13];
  float reals[19];
  std::memcpy(ints, b, sizeof(ints));
  std::memcpy(reals, b + sizeof(ints), sizeof(reals));
  int64_t *io[13] = {&h.nplocal, &h.npglobal, &h.izipx, &h.izipv, &h.image, &h.nn, &h.nnt,
                     &h.nt, &h.ncell, &h.ncb, &h.timestep, &h.cur_checkpoint, &h.cur_halofind};
  float *ro[19] = {&h.a,       &h.t,       &h.tau,       &h.dt_pp,     &h.dt_pm3,   &h.dt_pm2, &h.dt_pm1,
                   &h.dt_vmax, &h.mass_p_cdm, &h.box,    &h.h0,        &h.omega_m,  &h.omega_l, &h.s8,
                   &h.vsim2phys, &h.sigma_vres, &h.sigma_vi, &h.z_i,   &h.vz_max};
  for (int i = 0; i < 13; i++) *io[i] = ints[i];
  for (int i = 0; i < 19; i++) *ro[i] = reals[i];
}

static int write_file(const std::string &path, const void *data, size_t bytes) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return CUBE_ERR_INVALID;
  const size_t w = bytes ? std::fwrite(data, 1, bytes, f) : 0;
  const int c = std::fclose(f);
  return (w == bytes && c == 0) ? CUBE_OK : CUBE_ERR_INVALID;
}

static int read_file(const std::string &path, void *data, size_t bytes) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return CUBE_ERR_INVALID;
  const size_t r = bytes ? std::fread(data, 1, bytes, f) : 0;
  std::fclose(f);
  return r == bytes ? CUBE_OK : CUBE_ERR_INVALID;
}

int snapshot_write(const Lay &L, const char *prefix, const char *suffix, const cube_sim_header *h,
                   const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp, const float *vp,
                   const int64_t *pid) {
  if (!prefix || !suffix || !h || !rhoc || !idx_b_r) return CUBE_ERR_INVALID;
  const int nt = L.nt, ncb = L.ncb, nte = L.nte, ntile = L.ntile;
  // physical particles, tile by tile, row (k, j) by row: in a row the physical cells are
  // contiguous, after the ncb buffer cells on the left
  std::vector<int32_t> np_phys((size_t)ntile * nt * nt * nt);
  std::vector<int64_t> runs;  // (start, count) per physical row
  int64_t total = 0;
  for (int t = 0; t < ntile; t++)
    for (int k = 0; k < nt; k++)
      for (int j = 0; j < nt; j++) {
        const int64_t row = ((int64_t)t * nte + (k + ncb)) * nte + (j + ncb);
        const int32_t *r = rhoc + row * nte;
        int64_t after = 0;
        for (int i = ncb + nt; i < nte; i++) after += r[i];
        int64_t phys = 0;
        for (int i = 0; i < nt; i++) {
          if (r[ncb + i] < 0) return CUBE_ERR_INVALID;
          phys += r[ncb + i];
          np_phys[(((size_t)t * nt + k) * nt + j) * nt + i] = r[ncb + i];
        }
        const int64_t start = idx_b_r[row] - after - phys;
        if (start < 0) return CUBE_ERR_INVALID;
        if (phys) {
          runs.push_back(start);
          runs.push_back(phys);
        }
        total += phys;
      }
  if (total > 0 && (!xp || !vp)) return CUBE_ERR_INVALID;
  cube_sim_header hh = *h;
  hh.nplocal = total;
  unsigned char hb[kSimHeaderBytes];
  header_to_bytes(hh, hb);
  const std::string pre(prefix), suf(suffix);
  int s = write_file(pre + "info" + suf, hb, sizeof(hb));
  if (s != CUBE_OK) return s;
  std::vector<int16_t> bx((size_t)total * 3);
  std::vector<float> bv((size_t)total * 3);
  std::vector<int64_t> bp(pid ? (size_t)total : 0);
  int64_t o = 0;
  for (size_t q = 0; q < runs.size(); q += 2) {
    const int64_t a = runs[q], n = runs[q + 1];
    std::memcpy(&bx[3 * o], xp + 3 * a, sizeof(int16_t) * 3 * n);
    std::memcpy(&bv[3 * o], vp + 3 * a, sizeof(float) * 3 * n);
    if (pid) std::memcpy(&bp[o], pid + a, sizeof(int64_t) * n);
    o += n;
  }
  if ((s = write_file(pre + "xp" + suf, bx.data(), sizeof(int16_t) * bx.size())) != CUBE_OK) return s;
  if ((s = write_file(pre + "vp" + suf, bv.data(), sizeof(float) * bv.size())) != CUBE_OK) return s;
  if ((s = write_file(pre + "np" + suf, np_phys.data(), sizeof(int32_t) * np_phys.size())) != CUBE_OK) return s;
  if (pid && (s = write_file(pre + "id" + suf, bp.data(), sizeof(int64_t) * bp.size())) != CUBE_OK) return s;
  return CUBE_OK;
}

int snapshot_read(const Lay &L, const char *prefix, const char *suffix, cube_sim_header *h, int32_t *rhoc_phys,
                  int16_t *xp, float *vp, int64_t *pid, int64_t capacity) {
  if (!prefix || !suffix || !h) return CUBE_ERR_INVALID;
  const std::string pre(prefix), suf(suffix);
  unsigned char hb[kSimHeaderBytes];
  int s = read_file(pre + "info" + suf, hb, sizeof(hb));
  if (s != CUBE_OK) return s;
  header_from_bytes(hb, *h);
  // particle_initialization.f90:31-35: the stored formats must be the ones this build reads
  if (h->izipx != 2 || h->izipv != 2) return CUBE_ERR_INVALID;
  if (h->nnt != L.nnt || h->nt != L.nt || h->nplocal < 0) return CUBE_ERR_INVALID;
  if (h->nplocal > capacity) return CUBE_ERR_CAPACITY;
  const size_t n = (size_t)h->nplocal;
  if (n && (!xp || !vp)) return CUBE_ERR_INVALID;
  if (rhoc_phys &&
      (s = read_file(pre + "np" + suf, rhoc_phys, sizeof(int32_t) * (size_t)L.ntile * L.nt * L.nt * L.nt)) != CUBE_OK)
    return s;
  if (n && (s = read_file(pre + "xp" + suf, xp, sizeof(int16_t) * 3 * n)) != CUBE_OK) return s;
  if (n && (s = read_file(pre + "vp" + suf, vp, sizeof(float) * 3 * n)) != CUBE_OK) return s;
  if (pid && n && (s = read_file(pre + "id" + suf, pid, sizeof(int64_t) * n)) != CUBE_OK) return s;
  return CUBE_OK;
}

}  // namespace cube
