// C-ABI of the library: the reference-named entry points bound by kick.f90:12-46
// and finalize.f90:8-13, their status-returning variants, the fused kick and
// the inspection calls.  Owns the device context (buffers grown on demand and
// kept between kicks, cuFFT plans, Green tables), like the reference's static
// workspaces (pp_force_kernel.cu:467-494, pm3_fft_cuda.cu:56-71), but never
// aborts: every failure becomes a status code.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace cube {

static thread_local int t_last_error = CUBE_OK;

struct Buf {
  void *p = nullptr;
  size_t cap = 0;
};

struct GreenEntry {
  int n;
  float apm_soft, apm_range, gridsize;
  int p;
  float *d;
};

struct HostGreen {  // caller's table cached by pointer and size (pm3_fft_cuda.cu:153-175)
  const float *host;
  size_t count;
  float *d;
};

struct Plan {
  int n, batch;
  cufftType type;
  cufftHandle h;
  int pad = 0;   // C2R into the interior of arrays with `pad` ghost points per side
  int rank = 3;  // 3: whole meshes; 2: the x-y planes of meshes (batch = planes)
};

struct Ctx {
  bool configured = false;
  cube_layout pub{};
  Lay L{};
  int device = -1;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  // Host entry points upload vp on `copy` while PM3 runs; the compute stream waits on
  // vp_ready just before the first kernel that reads vp (the PM3 gather or the PP force).
  cudaStream_t copy = nullptr;
  cudaEvent_t vp_ready = nullptr;
  bool vp_pending = false;
  // The PP binning and work list run on `side`, beside PM3 on the compute stream.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Host kicks pipeline groups of consecutive tiles (one tile per group up to kPipeGroups
  // tiles; more groups cost more small launches than they overlap on a 512-tile batch):
  // group k holds tiles [grp_lo[k], grp_lo[k + 1])
  static constexpr int kMaxTileEvents = 64;
  static constexpr int kPipeGroups = 16;
  static_assert(kPipeGroups <= kMaxTileEvents, "one event of each kind per group");
  int ngrp = 0;
  int grp_lo[kMaxTileEvents + 1] = {};
  int grp_order[kMaxTileEvents] = {};  // host kicks: groups by decreasing particle count (the
                                       // order of vp uploads, gathers, PP launches and copies back)
  cudaEvent_t ev_tile[kMaxTileEvents] = {};  // per-group PP force done (host kicks)
  cudaEvent_t ev_copied = nullptr;           // last per-group vp copy enqueued
  bool vp_copied = false;                    // this host kick's vp is already on its way back
  // Host kicks upload xp group by group on `copy`; the deposit of a group waits only for its
  // own part (and so does the binning of a spill-free layout), everything else that reads xp
  // waits for all of it.
  cudaEvent_t ev_xp[kMaxTileEvents] = {};
  bool xp_pending = false;
  int xp_tiles = 0;  // groups uploaded
  // ... and vp group by group too: the PM3 gather of a group waits for its vp, and the PP force
  // of a group (on side or side2) waits for that group's gather (ev_ready) and the binning.
  cudaEvent_t ev_vp[kMaxTileEvents] = {}, ev_ready[kMaxTileEvents] = {};
  int vp_tiles = 0;          // > 0: vp was uploaded in this many group parts
  bool ready_tiles = false;  // ev_ready[k] recorded by this kick's PM3
  cudaStream_t side2 = nullptr;
  cudaEvent_t ev_pm3done = nullptr, ev_join2 = nullptr;
  Buf xp, rhoc, idx, vp, cell_base;
  Buf tiles, count, cell_start, scan_tmp, spos, spill, spill_rank, counters, items, range_loc, sched;
  Buf rho, rhok, force, jobs, out;
  Buf mlp_pos, mlp_rho;  // learned shell: positions of the stored copies, fine-grid CIC density
  // PP kernel shape: fixed (pp_fixed >= 0, cube_pp_set_shape) or autotuned, keyed by
  // pp_shape_key; pp_ms holds the last tuning's times, pp_last the shape of the last PP kick
  int pp_fixed = -1;
  std::unordered_map<uint64_t, int> pp_tuned;
  float pp_ms[kMaxPPShapes];
  int pp_last = 0;
  Ctx() {
    for (float &m : pp_ms) m = -1.0f;
  }
  Buf pp_scratch;  // tuning runs kick these velocities, not the caller's
  // drift and buffer rebuild scratch
  Buf dr_cb, dr_cb_new, dr_runrank, dr_run_base, dr_runs, dr_ctr, dr_dest_runs, dr_dest_start, dr_scan_tmp,
      dr_cursor, dr_phys, dr_list, dr_off, dr_rows, dr_total;
  Buf dh_rhoc, dh_idx, dh_xp, dh_vp, dh_pid, dh_rhoc2, dh_idx2, dh_xp2, dh_vp2, dh_pid2;  // host-array drift
  Buf pw_grid, pw_k, pw_bins;  // power spectrum
  Buf ks_out;                  // FP64 conservation sums
  Buf fb_out;                  // learned-shell fallback statistics
  Buf phi_pad;                 // padded potential of the brick kernels
  Buf brick_ctr;               // their work counter
  Buf dep_items;               // the brick deposit's work list
  cudaEvent_t tune_ev[2 * kMaxPPShapes] = {};
  void *h_stage = nullptr;  // pinned staging for small tables
  size_t h_stage_cap = 0;
  float *h_out = nullptr;   // pinned [8]: out[5], err
  std::vector<GreenEntry> greens;
  std::vector<HostGreen> hgreens;
  std::vector<Plan> plans;
  // Stage events of the last kRing timed calls.  Per call: 0 start, 1 after PM3,
  // 2 PP start, 3 PP force kernel start, 4 after the PP force kernel, 5 end, 6 after the PP
  // work list.  The PP binning and work list (2 to 6) may run beside PM3 (0 to 1).
  static constexpr int kRing = 256;
  cudaEvent_t ring[kRing][7] = {};
  bool ring_pm3[kRing] = {}, ring_pp[kRing] = {};
  int ring_cur = 0, ring_next = 0, ring_count = 0;
  bool timing = false;
  float stage_ms[4] = {0, 0, 0, 0};
  long long launches = 0;  // kernels of this library enqueued so far
  // Pinned staging areas for the small per-call tables, used round robin so the
  // host can enqueue the next kick while earlier ones still copy out of theirs.
  static constexpr int kStage = 4;
  // a captured graph's own staging area, used instead of the ring while it is captured
  void *stage_override = nullptr;
  size_t stage_override_cap = 0;
  void *stage_buf[kStage] = {};
  cudaEvent_t stage_evs[kStage] = {};
  bool stage_used[kStage] = {};
  int stage_slot = 0;
};

static Ctx g;
static std::mutex g_mu;

static int fail(int code) {
  t_last_error = code;
  return code;
}

#define CU(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      if (getenv("CUBE_VERBOSE"))                                                      \
        fprintf(stderr, "cube2_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return fail(CUBE_ERR_CUDA);                                                      \
    }                                                                                  \
  } while (0)

#define CF(x)                                                                          \
  do {                                                                                 \
    cufftResult r_ = (x);                                                              \
    if (r_ != CUFFT_SUCCESS) {                                                         \
      if (getenv("CUBE_VERBOSE")) fprintf(stderr, "cube2_b200: %s failed: %d\n", #x, (int)r_); \
      return fail(CUBE_ERR_CUFFT);                                                     \
    }                                                                                  \
  } while (0)

#define CK(x)                    \
  do {                           \
    int s_ = (x);                \
    if (s_ != CUBE_OK) return s_; \
  } while (0)

static int grow(Buf &b, size_t bytes) {
  if (bytes <= b.cap) return CUBE_OK;
  size_t want = std::max(bytes, b.cap + b.cap / 4);
  if (b.p) {
    CU(cudaStreamSynchronize(g.stream));
    CU(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
  }
  CU(cudaMalloc(&b.p, want));
  b.cap = want;
  return CUBE_OK;
}

static void release(Buf &b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

// Device binding per process, as c_select_gpu_for_image (pp_force_kernel.cu:80-128)
// does: the node-local rank picks the device when several are visible.
static int local_rank() {
  const char *vars[] = {"MPI_LOCALRANKID", "OMPI_COMM_WORLD_LOCAL_RANK", "SLURM_LOCALID", "PMI_LOCAL_RANK",
                        "LOCAL_RANK"};
  for (const char *v : vars) {
    const char *s = getenv(v);
    if (s) return atoi(s);
  }
  return 0;
}

static int ensure_device() {
  if (g.device >= 0) {
    CU(cudaSetDevice(g.device));
    return CUBE_OK;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) return fail(CUBE_ERR_NO_DEVICE);
  const int dev = count == 1 ? 0 : local_rank();
  if (dev < 0 || dev >= count) return fail(CUBE_ERR_NO_DEVICE);
  CU(cudaSetDevice(dev));
  g.device = dev;
  CU(cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, dev));
  CU(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
  CU(cudaStreamCreateWithFlags(&g.copy, cudaStreamNonBlocking));
  CU(cudaEventCreateWithFlags(&g.vp_ready, cudaEventDisableTiming));
  CU(cudaStreamCreateWithFlags(&g.side, cudaStreamNonBlocking));
  CU(cudaEventCreateWithFlags(&g.ev_fork, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&g.ev_join, cudaEventDisableTiming));
  for (auto &e : g.ev_tile) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : g.ev_xp) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : g.ev_vp) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : g.ev_ready) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  CU(cudaStreamCreateWithFlags(&g.side2, cudaStreamNonBlocking));
  CU(cudaEventCreateWithFlags(&g.ev_pm3done, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&g.ev_join2, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&g.ev_copied, cudaEventDisableTiming));
  CU(cudaMallocHost(&g.h_out, sizeof(float) * 8));
  for (auto &slot : g.ring)
    for (auto &e : slot) CU(cudaEventCreate(&e));
  for (auto &e : g.stage_evs) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return CUBE_OK;
}

// Make every staging area hold `bytes` and select the next one, waiting until
// the call that last used it has finished copying out of it.
static int stage_begin(size_t bytes) {
  if (g.stage_override) {
    if (bytes > g.stage_override_cap) return fail(CUBE_ERR_CAPACITY);
    g.h_stage = g.stage_override;
    return CUBE_OK;
  }
  if (bytes > g.h_stage_cap) {
    CU(cudaDeviceSynchronize());
    for (auto &b : g.stage_buf)
      if (b) CU(cudaFreeHost(b));
    g.h_stage_cap = std::max(bytes, (size_t)1 << 20);
    for (auto &b : g.stage_buf) CU(cudaMallocHost(&b, g.h_stage_cap));
    for (auto &u : g.stage_used) u = false;
  }
  const int s = g.stage_slot;
  if (g.stage_used[s]) {
    CU(cudaEventSynchronize(g.stage_evs[s]));
    g.stage_used[s] = false;
  }
  g.h_stage = g.stage_buf[s];
  return CUBE_OK;
}

// Mark the current staging area busy until the stream passes this point.
static int stage_end() {
  if (g.stage_override) return CUBE_OK;
  const int s = g.stage_slot;
  CU(cudaEventRecord(g.stage_evs[s], g.stream));
  g.stage_used[s] = true;
  g.stage_slot = (s + 1) % Ctx::kStage;
  return CUBE_OK;
}

// upload a small host table through the pinned staging area (offset in bytes)
template <class T>
static int upload(Buf &dst, const T *src, size_t count, size_t &stage_off, cudaStream_t st = nullptr) {
  const size_t bytes = sizeof(T) * count;
  CK(grow(dst, bytes > 0 ? bytes : 16));
  if (!bytes) return CUBE_OK;
  stage_off = (stage_off + 255) & ~(size_t)255;
  if (stage_off + bytes > (g.stage_override ? g.stage_override_cap : g.h_stage_cap)) return fail(CUBE_ERR_CAPACITY);
  memcpy((char *)g.h_stage + stage_off, src, bytes);
  CU(cudaMemcpyAsync(dst.p, (char *)g.h_stage + stage_off, bytes, cudaMemcpyHostToDevice, st ? st : g.stream));
  stage_off += bytes;
  return CUBE_OK;
}

// order stream `st` after the pending upload of tile t's xp (t < 0: all of xp)
static int wait_xp(cudaStream_t st, int t = -1) {
  if (!g.xp_pending) return CUBE_OK;
  CU(cudaStreamWaitEvent(st, g.ev_xp[t < 0 ? g.xp_tiles - 1 : t], 0));
  return CUBE_OK;
}

// order the compute stream after a pending vp upload
static int wait_vp() {
  if (!g.vp_pending) return CUBE_OK;
  // the group parts go up in grp_order: the last one recorded covers them all
  CU(cudaStreamWaitEvent(g.stream, g.vp_tiles ? g.ev_vp[g.grp_order[g.vp_tiles - 1]] : g.vp_ready, 0));
  g.vp_pending = false;
  return CUBE_OK;
}

// Two-dimensional transforms of `batch` consecutive x-y planes of side n: R2C from real planes
// of n^2 points to half-spectrum planes of n (n/2 + 1); C2R back, into planes of n^2 points or,
// with pad > 0, into the interior rows of planes of (n + 2 pad)^2 points.
static int get_plan2d(int n, int batch, cufftType type, int pad, cufftHandle *out) {
  for (auto &p : g.plans)
    if (p.rank == 2 && p.n == n && p.batch == batch && p.type == type && p.pad == pad) {
      CF(cufftSetStream(p.h, g.stream));
      *out = p.h;
      return CUBE_OK;
    }
  Plan p{n, batch, type, 0, pad, 2};
  const int h = n / 2 + 1, m = n + 2 * pad;
  int dims[2] = {n, n}, real[2] = {m, m}, cplx[2] = {n, h};
  if (type == CUFFT_R2C) {
    CF(cufftPlanMany(&p.h, 2, dims, real, 1, m * m, cplx, 1, n * h, CUFFT_R2C, batch));
  } else {
    CF(cufftPlanMany(&p.h, 2, dims, cplx, 1, n * h, real, 1, m * m, CUFFT_C2R, batch));
  }
  CF(cufftSetStream(p.h, g.stream));
  g.plans.push_back(p);
  *out = p.h;
  return CUBE_OK;
}

// C2R whose output lands in the interior of [batch][(n+2 pad)^3] arrays (advanced layout)
static int get_plan_padded_c2r(int n, int batch, int pad, cufftHandle *out) {
  for (auto &p : g.plans)
    if (p.rank == 3 && p.n == n && p.batch == batch && p.type == CUFFT_C2R && p.pad == pad) {
      CF(cufftSetStream(p.h, g.stream));
      *out = p.h;
      return CUBE_OK;
    }
  Plan p{n, batch, CUFFT_C2R, 0, pad};
  const int m = n + 2 * pad;
  int dims[3] = {n, n, n}, inembed[3] = {n, n, n / 2 + 1}, onembed[3] = {m, m, m};
  CF(cufftPlanMany(&p.h, 3, dims, inembed, 1, n * n * (n / 2 + 1), onembed, 1, m * m * m, CUFFT_C2R, batch));
  CF(cufftSetStream(p.h, g.stream));
  g.plans.push_back(p);
  *out = p.h;
  return CUBE_OK;
}

static int get_plan(int n, int batch, cufftType type, cufftHandle *out) {
  for (auto &p : g.plans)
    if (p.rank == 3 && p.n == n && p.batch == batch && p.type == type && p.pad == 0) {
      CF(cufftSetStream(p.h, g.stream));
      *out = p.h;
      return CUBE_OK;
    }
  Plan p{n, batch, type, 0};
  int dims[3] = {n, n, n};
  CF(cufftPlanMany(&p.h, 3, dims, nullptr, 1, 0, nullptr, 1, 0, type, batch));
  CF(cufftSetStream(p.h, g.stream));
  g.plans.push_back(p);
  *out = p.h;
  return CUBE_OK;
}

// ---------------------------------------------------------------------------------------------
// metadata

struct Meta {
  std::vector<int> ires_loc, owner;  // by subtile location
  std::vector<float> range_loc;
  std::vector<TilePP> tiles;
  int64_t ncells = 0;
  int max_rcp = 1;
};

static inline int loc_of(const Lay &L, int sx, int sy, int sz, int tx, int ty, int tz) {
  return (((tz * L.nnt + ty) * L.nnt + tx) * L.nns + sz) * L.nns * L.nns + sy * L.nns + sx;
}

// validate and reorder the per-subtile tables by location (pp_force_kernel.cu:987-1004)
static int build_meta(const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf, const float *apm3,
                      Meta &m) {
  const Lay &L = g.L;
  if (!ires || !ixyz3 || !ratio_sf) return fail(CUBE_ERR_INVALID);
  m.ires_loc.assign(L.ns3, -1);
  m.owner.assign(L.ns3, -1);
  m.range_loc.assign(L.ns3, 0.f);
  for (int it = 0; it < L.ns3; it++) {
    const int *r = ixyz3 + 6 * it;
    const int sx = r[0] - 1, sy = r[1] - 1, sz = r[2] - 1, tx = r[3] - 1, ty = r[4] - 1, tz = r[5] - 1;
    if (sx < 0 || sx >= L.nns || sy < 0 || sy >= L.nns || sz < 0 || sz >= L.nns || tx < 0 || tx >= L.nnt ||
        ty < 0 || ty >= L.nnt || tz < 0 || tz >= L.nnt || ires[it] < 2 || ires[it] > 6)
      return fail(CUBE_ERR_INVALID);
    const int loc = loc_of(L, sx, sy, sz, tx, ty, tz);
    if (m.owner[loc] >= 0) return fail(CUBE_ERR_INVALID);
    m.ires_loc[loc] = ires[it];
    m.owner[loc] = it;
    if (apm3) m.range_loc[loc] = apm3[ires[it] - 1];
  }
  for (int l = 0; l < 7; l++)
    if (ratio_sf[l] < 1 || ratio_sf[l] > 64) return fail(CUBE_ERR_INVALID);
  m.tiles.resize(L.ntile);
  int64_t cell0 = 0;
  m.max_rcp = 1;
  for (int t = 0; t < L.ntile; t++) {
    int rcp = ratio_sf[1];
    const int nss = L.nns * L.nns * L.nns;
    for (int q = 0; q < nss; q++) rcp = std::max(rcp, ratio_sf[m.ires_loc[t * nss + q] - 1]);
    TilePP tp;
    tp.rcp = rcp;
    tp.S = rcp * (L.nt + 2);
    tp.cell0 = cell0;
    cell0 += (int64_t)tp.S * tp.S * tp.S;
    m.tiles[t] = tp;
    m.max_rcp = std::max(m.max_rcp, rcp);
  }
  m.ncells = cell0;
  if (m.ncells >= ((int64_t)1 << 31)) return fail(CUBE_ERR_CAPACITY);
  return CUBE_OK;
}

// particles kicked per subtile = particles of its interior coarse cells (pm3_fft_cuda.cu:437,
// pp_force_kernel.cu:705-710), written by subtile index it
static void fill_ptotal(const Meta &m, const int32_t *rhoc, double *ptotal) {
  const Lay &L = g.L;
  for (int loc = 0; loc < L.ns3; loc++) {
    const int nss = L.nns * L.nns * L.nns;
    const int t = loc / nss, s = loc % nss;
    const int sx = s % L.nns, sy = (s / L.nns) % L.nns, sz = s / (L.nns * L.nns);
    double c = 0;
    for (int k = 0; k < L.ntt; k++)
      for (int j = 0; j < L.ntt; j++)
        for (int i = 0; i < L.ntt; i++) {
          const int ci = L.ncb + sx * L.ntt + i, cj = L.ncb + sy * L.ntt + j, ck = L.ncb + sz * L.ntt + k;
          c += rhoc[(((int64_t)t * L.nte + ck) * L.nte + cj) * L.nte + ci];
        }
    ptotal[m.owner[loc]] = c;
  }
}

// ---------------------------------------------------------------------------------------------
// pipeline stages (device pointers in ctx buffers or caller's)

struct Dev {
  const int16_t *xp;
  const int32_t *rhoc;
  const int64_t *idx;
  float *vp;
  int64_t n_used;
  // host kicks only: the caller's vp and spine; each group's vp is copied back as soon as
  // that group's PP force kernel has finished
  float *h_vp = nullptr;
  const int64_t *h_idx = nullptr;
};

static int get_green_periodic(int n, int rsf, float **out) {
  const Lay &L = g.L;
  const float gs = 1.0f / (float)rsf;
  for (auto &e : g.greens)
    if (e.n == n && e.apm_soft == L.apm3f && e.apm_range == L.apm_range && e.gridsize == gs && e.p == L.p_order) {
      *out = e.d;
      return CUBE_OK;
    }
  GreenEntry e{n, L.apm3f, L.apm_range, gs, L.p_order, nullptr};
  CU(cudaMalloc(&e.d, sizeof(float) * (size_t)n * n * (n / 2 + 1)));
  launch_green_fp64(n, L.apm3f, L.apm_range, gs, L.p_order, e.d, g.stream);
  CU(cudaGetLastError());
  g.greens.push_back(e);
  *out = e.d;
  return CUBE_OK;
}

// Green table of any mesh, tabulated on the device in FP64 and kept by its parameters
static int get_green_params(int n, float apm_soft, float apm_range, float gridsize, float **out) {
  for (auto &e : g.greens)
    if (e.n == n && e.apm_soft == apm_soft && e.apm_range == apm_range && e.gridsize == gridsize &&
        e.p == g.L.p_order) {
      *out = e.d;
      return CUBE_OK;
    }
  GreenEntry e{n, apm_soft, apm_range, gridsize, g.L.p_order, nullptr};
  CU(cudaMalloc(&e.d, sizeof(float) * (size_t)n * n * (n / 2 + 1)));
  launch_green_fp64(n, apm_soft, apm_range, gridsize, g.L.p_order, e.d, g.stream);
  CU(cudaGetLastError());
  g.greens.push_back(e);
  *out = e.d;
  return CUBE_OK;
}

static int get_green_host(const float *host, int n, float **out) {
  const size_t count = (size_t)n * n * (n / 2 + 1);
  for (auto &e : g.hgreens)
    if (e.host == host && e.count == count) {
      *out = e.d;
      return CUBE_OK;
    }
  HostGreen e{host, count, nullptr};
  CU(cudaMalloc(&e.d, sizeof(float) * count));
  CU(cudaMemcpy(e.d, host, sizeof(float) * count, cudaMemcpyHostToDevice));
  g.hgreens.push_back(e);
  *out = e.d;
  return CUBE_OK;
}

static const int kFftBuckets[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512};

static int run_pm3(const Meta &m, const int32_t *ires, const int32_t *ratio_sf, const float *const *gk,
                   const Dev &d, float mass, float kick, bool want_vmax, size_t &soff) {
  const Lay &L = g.L;
  if (L.pm3_mode == CUBE_PM3_PERIODIC || L.pm3_mode == CUBE_PM3_TILE_PERIODIC) {
    // one periodic mesh over the image, or one per parent tile (each tile its own periodic box)
    const bool per_tile = L.pm3_mode == CUBE_PM3_TILE_PERIODIC;
    const int rsf = ratio_sf[m.ires_loc[0] - 1];
    for (int q = 0; q < L.ns3; q++)
      if (ratio_sf[m.ires_loc[q] - 1] != rsf) return fail(CUBE_ERR_INVALID);
    const int n = (per_tile ? L.nt * L.rcs : L.ng) * rsf;
    const int nslots = per_tile ? L.ntile : 1;
    const int64_t n3 = (int64_t)n * n * n, nk = (int64_t)n * n * (n / 2 + 1);
    float *G = nullptr;
    CK(get_green_periodic(n, rsf, &G));
    CK(grow(g.rho, sizeof(float) * n3 * nslots));
    CK(grow(g.rhok, sizeof(cufftComplex) * nk * nslots));
    const double scale = (double)L.rcs / (double)(1.0f / (float)rsf);
    std::vector<MeshJob> jobs(L.ntile);
    for (int t = 0; t < L.ntile; t++) {
      const int tx = t % L.nnt, ty = (t / L.nnt) % L.nnt, tz = t / (L.nnt * L.nnt);
      MeshJob &J = jobs[t];
      J.t = t;
      J.slot = per_tile ? t : 0;
      J.range = 0.f;
      const int tc[3] = {tx, ty, tz};
      for (int q = 0; q < 3; q++) {
        J.lo[q] = L.ncb;
        J.alo[q] = L.ncb;
        J.off[q] = per_tile ? 0.0 : -(double)tc[q] * L.nt * scale;
      }
    }
    CK(upload(g.jobs, jobs.data(), jobs.size(), soff));
    PM3Args a{};
    a.L = &g.L;
    a.rsf = rsf;
    a.n = n;
    a.nslots = nslots;
    a.jobs = (const MeshJob *)g.jobs.p;
    a.njobs = L.ntile;
    for (int q = 0; q < 3; q++) a.rdep[q] = a.ract[q] = L.nt;
    a.wrap = 1;
    a.shift = 0;
    a.fphys_lo = 0;
    a.fphys_n = n;
    a.scale = scale;
    a.xp = d.xp;
    a.rhoc = d.rhoc;
    a.cell_base = (const int64_t *)g.cell_base.p;
    a.rho = (float *)g.rho.p;
    a.rhok = (cufftComplex *)g.rhok.p;
    a.force = nullptr;
    a.green = G;
    a.mass = mass;
    a.kick = kick;
    a.vp = d.vp;
    a.out = (float *)g.out.p;
    a.want_vmax = want_vmax;
    a.err = (int32_t *)g.counters.p + 2;
    a.num_sms = g.num_sms;
    // the force difference is fused into the gather brick by brick where the geometry allows;
    // otherwise the three force arrays are written and gathered from
    const bool fused = pm3_brick_mc(a) > 0;
    const int64_t m3 = (int64_t)(n + 2 * kPotPad) * (n + 2 * kPotPad) * (n + 2 * kPotPad);
    if (!fused) {
      CK(grow(g.force, sizeof(float) * n3 * 3 * nslots));
      a.force = (float *)g.force.p;
    } else {
      CK(grow(g.phi_pad, sizeof(float) * m3 * nslots));
      a.phi_pad = (float *)g.phi_pad.p;
      CK(grow(g.brick_ctr, sizeof(int32_t) * 64));
      a.brick_ctr = (int32_t *)g.brick_ctr.p;
    }
    {
      CK(grow(g.dep_items, pm3_dep_items_bytes((int64_t)a.rdep[0] * a.rdep[1] * a.rdep[2], a.njobs, d.n_used)));
      a.dep_items = (int2 *)g.dep_items.p;
      a.n_particles_hint = d.n_used;
    }
    // k-space step: two-dimensional transforms of the x-y planes around the fused z step where
    // the mesh side allows, otherwise three-dimensional transforms around the Green multiply.
    // Several padded meshes (one per tile) take the three-dimensional path: their planes are
    // not equally spaced, and one plane C2R call per mesh costs more than it saves.
    const bool zsplit = pm3_kspace_z_ok(n) && (!fused || nslots == 1);
    cufftHandle fw, bw;
    if (zsplit) {
      CK(get_plan2d(n, n * nslots, CUFFT_R2C, 0, &fw));
      CK(get_plan2d(n, fused ? n : n * nslots, CUFFT_C2R, fused ? kPotPad : 0, &bw));
    } else {
      CK(get_plan(n, nslots, CUFFT_R2C, &fw));
      if (fused) CK(get_plan_padded_c2r(n, nslots, kPotPad, &bw));
      else CK(get_plan(n, nslots, CUFFT_C2R, &bw));
    }
    CU(cudaMemsetAsync(g.rho.p, 0, sizeof(float) * n3 * nslots, g.stream));
    if (g.xp_pending) {  // deposit each group of tiles as soon as its particles are on the device
      PM3Args at = a;
      for (int k = 0; k < g.ngrp; k++) {
        CK(wait_xp(g.stream, k));
        at.jobs = (const MeshJob *)g.jobs.p + g.grp_lo[k];
        at.njobs = g.grp_lo[k + 1] - g.grp_lo[k];
        g.launches += launch_pm3_deposit(at, g.stream);
      }
    } else {
      g.launches += launch_pm3_deposit(a, g.stream);
    }
    CF(cufftExecR2C(fw, (cufftReal *)g.rho.p, (cufftComplex *)g.rhok.p));
    if (zsplit) launch_pm3_kspace_z(a, g.stream);
    else launch_pm3_kspace(a, g.stream);
    if (fused) {
      // the potential into the interior of the padded array, then its periodic ghost points
      const int64_t mm = n + 2 * kPotPad;
      float *interior = a.phi_pad + (kPotPad * mm + kPotPad) * mm + kPotPad;
      if (zsplit) {  // plane transforms, one mesh at a time (the padded meshes are m^3 apart)
        for (int sl = 0; sl < nslots; sl++)
          CF(cufftExecC2R(bw, (cufftComplex *)g.rhok.p + (int64_t)sl * nk, (cufftReal *)(interior + sl * mm * mm * mm)));
      } else {
        CF(cufftExecC2R(bw, (cufftComplex *)g.rhok.p, (cufftReal *)interior));
      }
      launch_pm3_ghosts(a, g.stream);
    } else {
      CF(cufftExecC2R(bw, (cufftComplex *)g.rhok.p, (cufftReal *)g.rho.p));  // potential
      launch_pm3_force(a, g.stream);
    }
    auto gather = [&](const PM3Args &ga) {
      if (fused) launch_pm3_force_gather(ga, g.stream);
      else launch_pm3_gather(ga, g.stream);
    };
    if (g.vp_pending && g.vp_tiles == g.ngrp && g.ngrp > 0) {  // gather each group once its vp is in
      PM3Args at = a;
      for (int kk = 0; kk < g.ngrp; kk++) {
        const int k = g.grp_order[kk];
        CU(cudaStreamWaitEvent(g.stream, g.ev_vp[k], 0));
        at.jobs = (const MeshJob *)g.jobs.p + g.grp_lo[k];
        at.njobs = g.grp_lo[k + 1] - g.grp_lo[k];
        gather(at);
        CU(cudaEventRecord(g.ev_ready[k], g.stream));
      }
      g.vp_pending = false;
      g.ready_tiles = true;
      g.launches += g.ngrp - 1;
    } else {
      CK(wait_vp());
      gather(a);
    }
    g.launches += 3;  // k-space, then ghosts + force-gather or force + gather
    CU(cudaGetLastError());
    return CUBE_OK;
  }
  // buffered subtile meshes grouped by level (pm3_fft_cuda.cu:553-591)
  const size_t soff0 = soff;
  CK(wait_xp(g.stream));
  for (int lev = 2; lev <= 6; lev++) {
    std::vector<int> locs;
    for (int q = 0; q < L.ns3; q++)
      if (m.ires_loc[q] == lev) locs.push_back(q);
    if (locs.empty()) continue;
    if (!gk || !gk[lev - 2]) return fail(CUBE_ERR_INVALID);
    const int rsf = ratio_sf[lev - 1];
    const int nfp = L.ntt * L.rcs * rsf, nfb = L.rcs * rsf, n = nfp + 2 * nfb;
    const int64_t n3 = (int64_t)n * n * n, nk = (int64_t)n * n * (n / 2 + 1);
    float *G = nullptr;
    CK(get_green_host(gk[lev - 2], n, &G));
    const double scale = (double)L.rcs / (double)(1.0f / (float)rsf);
    const size_t per_slot = sizeof(float) * (size_t)n3 * 4 + sizeof(cufftComplex) * (size_t)nk;
    const size_t budget = (size_t)8 << 30;
    int bmax = (int)std::max<size_t>(1, budget / per_slot);
    bmax = std::min<int>(bmax, 512);
    for (size_t j0 = 0; j0 < locs.size(); j0 += bmax) {
      const int nj = (int)std::min<size_t>(bmax, locs.size() - j0);
      int nb = nj;
      for (int b : kFftBuckets)
        if (b >= nj) {
          nb = b;
          break;
        }
      CK(grow(g.rho, sizeof(float) * n3 * nb));
      CK(grow(g.rhok, sizeof(cufftComplex) * nk * nb));
      CK(grow(g.force, sizeof(float) * n3 * 3 * nb));
      std::vector<MeshJob> jobs(nj);
      for (int j = 0; j < nj; j++) {
        const int loc = locs[j0 + j];
        const int nss = L.nns * L.nns * L.nns;
        const int t = loc / nss, s = loc % nss;
        const int us[3] = {s % L.nns, (s / L.nns) % L.nns, s / (L.nns * L.nns)};
        MeshJob &J = jobs[j];
        J.t = t;
        J.slot = j;
        J.range = 0.f;
        for (int q = 0; q < 3; q++) {
          J.lo[q] = us[q] * L.ntt + L.ncb - 1;  // nc1 - nloop (kick.f90:429-432)
          J.alo[q] = us[q] * L.ntt + L.ncb;     // nc1 (kick.f90:503-505)
          J.off[q] = (double)us[q] * nfp;        // utile_shift * nfp (kick.f90:438)
        }
      }
      CK(upload(g.jobs, jobs.data(), jobs.size(), soff));
      PM3Args a{};
      a.L = &g.L;
      a.rsf = rsf;
      a.n = n;
      a.nslots = nb;
      a.jobs = (const MeshJob *)g.jobs.p;
      a.njobs = nj;
      for (int q = 0; q < 3; q++) {
        a.rdep[q] = L.ntt + 2;
        a.ract[q] = L.ntt;
      }
      a.wrap = 0;
      a.shift = nfb;
      a.fphys_lo = nfb;
      a.fphys_n = nfp;
      a.scale = scale;
      a.xp = d.xp;
      a.rhoc = d.rhoc;
      a.cell_base = (const int64_t *)g.cell_base.p;
      a.rho = (float *)g.rho.p;
      a.rhok = (cufftComplex *)g.rhok.p;
      a.force = (float *)g.force.p;
      a.green = G;
      a.mass = mass;
      a.kick = kick;
      a.vp = d.vp;
      a.out = (float *)g.out.p;
      a.want_vmax = want_vmax;
      cufftHandle fw, bw;
      CK(get_plan(n, nb, CUFFT_R2C, &fw));
      CK(get_plan(n, nb, CUFFT_C2R, &bw));
      CU(cudaMemsetAsync(g.rho.p, 0, sizeof(float) * n3 * nb, g.stream));
      launch_pm3_deposit(a, g.stream);
      CF(cufftExecR2C(fw, (cufftReal *)g.rho.p, (cufftComplex *)g.rhok.p));
      launch_pm3_kspace(a, g.stream);
      CF(cufftExecC2R(bw, (cufftComplex *)g.rhok.p, (cufftReal *)g.rho.p));  // potentials
      a.nslots = nj;  // force and f2max of the real jobs only
      launch_pm3_force(a, g.stream);
      CK(wait_vp());
      launch_pm3_gather(a, g.stream);
      g.launches += 4;
      CU(cudaGetLastError());
      // the job table is reused by the next batch
      CU(cudaStreamSynchronize(g.stream));
      soff = soff0;  // tables uploaded before PM3 (the PP grid) keep their staging slots
    }
  }
  return CUBE_OK;
}

static void fnv_mix(uint64_t &h, const void *data, size_t n) {
  const unsigned char *b = (const unsigned char *)data;
  for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
}

// What the fastest PP shape depends on: the layout's PP geometry, the per-tile PP grids, the PP
// ranges by subtile and the octave of the stored-particle count.
static uint64_t pp_shape_key(const Meta &m, int64_t n_used) {
  uint64_t h = 1469598103934665603ull;
  const int geo[6] = {g.L.ng, g.L.nnt, g.L.nns, g.L.rcs, g.L.ngb, 0};
  fnv_mix(h, geo, sizeof(geo));
  fnv_mix(h, &g.L.app, sizeof(float));
  for (const TilePP &t : m.tiles) fnv_mix(h, &t.rcp, sizeof(int));
  fnv_mix(h, m.range_loc.data(), sizeof(float) * m.range_loc.size());
  int octave = 0;
  while (octave < 63 && (n_used >> octave) > 1) octave++;
  fnv_mix(h, &octave, sizeof(int));
  return h;
}

// PP kernel shape for this kick (p.shape).  A fixed shape is used as is.  Otherwise the shape is
// looked up by pp_shape_key; on a miss every shape is timed on this kick's own binned particles
// (work list + force kernel, kicking scratch velocities), twice, and the fastest by the better of
// its two times is kept.  The binning has been enqueued on `st` already; the host waits for the
// timings, once per key.  A kick being captured into a graph cannot wait and uses shape 0.
static int choose_pp_shape(const Meta &m, int64_t n_used, PPArgs &p, cudaStream_t st) {
  if (g.pp_fixed >= 0) {
    p.shape = g.pp_last = g.pp_fixed;
    return CUBE_OK;
  }
  const uint64_t key = pp_shape_key(m, n_used);
  auto hit = g.pp_tuned.find(key);
  if (hit != g.pp_tuned.end()) {
    p.shape = g.pp_last = hit->second;
    return CUBE_OK;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  CU(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    p.shape = g.pp_last = 0;
    return CUBE_OK;
  }
  const int ns = pp_num_shapes();
  for (int k = 0; k < 2 * ns; k++)
    if (!g.tune_ev[k]) CU(cudaEventCreate(&g.tune_ev[k]));
  const size_t nv = 3 * (size_t)std::max<int64_t>(n_used, 1);
  CK(grow(g.pp_scratch, sizeof(float) * (nv + 8)));
  CU(cudaMemsetAsync(g.pp_scratch.p, 0, sizeof(float) * (nv + 8), st));
  PPArgs q = p;
  q.vp = (float *)g.pp_scratch.p;
  q.out = q.vp + nv;
  float best[kMaxPPShapes];
  for (int k = 0; k < ns; k++) best[k] = 3.0e38f;
  for (int rep = 0; rep < 2; rep++) {
    for (int k = 0; k < ns; k++) {
      q.shape = k;
      CU(cudaEventRecord(g.tune_ev[2 * k], st));
      launch_pp_items(q, st);
      launch_pp_force(q, st);
      CU(cudaEventRecord(g.tune_ev[2 * k + 1], st));
    }
    CU(cudaGetLastError());
    g.launches += 4 * ns;
    CU(cudaEventSynchronize(g.tune_ev[2 * ns - 1]));
    for (int k = 0; k < ns; k++) {
      float ms = 0;
      CU(cudaEventElapsedTime(&ms, g.tune_ev[2 * k], g.tune_ev[2 * k + 1]));
      best[k] = std::min(best[k], ms);
    }
  }
  int pick = 0;
  for (int k = 0; k < ns; k++) {
    g.pp_ms[k] = best[k];
    if (best[k] < best[pick]) pick = k;
  }
  g.pp_tuned[key] = pick;
  p.shape = g.pp_last = pick;
  return CUBE_OK;
}

// PP binning and work list on stream `st`; fills the arguments of the force kernel.  With
// `pairs` non-null the force kernel will only count accepted pairs and leave vp untouched.
static int run_pp_prep(const Meta &m, const Dev &d, float mass, float kick, size_t &soff, PPArgs &p,
                       cudaStream_t st, unsigned long long *pairs) {
  const Lay &L = g.L;
  CK(upload(g.tiles, m.tiles.data(), m.tiles.size(), soff, st));
  CK(upload(g.range_loc, m.range_loc.data(), m.range_loc.size(), soff, st));
  CK(grow(g.count, sizeof(int32_t) * (size_t)m.ncells));
  CK(grow(g.cell_start, sizeof(int32_t) * (size_t)(m.ncells + 1)));
  CK(grow(g.scan_tmp, sizeof(int32_t) * scan_tmp_elems(m.ncells)));
  CK(grow(g.spos, sizeof(float4) * (size_t)std::max<int64_t>(d.n_used, 1)));
  const int spill_cap = 2048;
  CK(grow(g.spill, sizeof(Spill) * spill_cap));
  CK(grow(g.spill_rank, sizeof(int32_t) * spill_cap));
  int64_t interior = 0;
  for (auto &t : m.tiles) interior += (int64_t)L.nt * t.rcp * L.nt * t.rcp * L.nt * t.rcp;
  const int64_t item_cap = interior + d.n_used / pp_min_chunk() + 16;
  CK(grow(g.items, sizeof(PPItem) * (size_t)item_cap));
  CK(grow(g.sched, sizeof(int32_t) * sched_ints(L.ntile)));
  int32_t *ctr = (int32_t *)g.counters.p;  // [0] spill_n [2] err
  BinArgs b{};
  b.L = &g.L;
  b.d_tiles = (const TilePP *)g.tiles.p;
  b.max_rcp = m.max_rcp;
  b.ncells = m.ncells;
  b.xp = d.xp;
  b.rhoc = d.rhoc;
  b.cell_base = (const int64_t *)g.cell_base.p;
  b.count = (int32_t *)g.count.p;
  b.cell_start = (int32_t *)g.cell_start.p;
  b.spos = (float4 *)g.spos.p;
  b.spill = (Spill *)g.spill.p;
  b.spill_rank = (int32_t *)g.spill_rank.p;
  b.spill_n = ctr + 0;
  b.spill_cap = spill_cap;
  b.scan_tmp = (int32_t *)g.scan_tmp.p;
  b.err = ctr + 2;
  if (bin_smem_bytes(m.max_rcp) > 200 * 1024) return fail(CUBE_ERR_INVALID);  // rcp^3 histograms per warp
  b.spatial = 1;
  if (g.xp_pending && pp_binning_spill_free(L, m.tiles.data())) {
    // xp is arriving group by group: each group of tiles is binned as soon as its xp is in
    if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][2], st));
    for (int k = 0; k < g.ngrp; k++) {
      CK(wait_xp(st, k));
      launch_pp_binning_tiles(b, m.tiles.data(), g.grp_lo[k], g.grp_lo[k + 1], st);
      g.launches += 5;  // count, 3 scan passes, scatter
    }
  } else {
    CK(wait_xp(st));
    if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][2], st));
    launch_pp_binning(b, st);
    g.launches += 7;  // count, spill sort, 3 scan passes, scatter, spill placement
  }
  CU(cudaGetLastError());
  p = PPArgs{};
  p.L = &g.L;
  p.d_tiles = (const TilePP *)g.tiles.p;
  p.h_tiles = m.tiles.data();
  p.ncells = m.ncells;
  p.cell_start = (const int32_t *)g.cell_start.p;
  p.spos = (const float4 *)g.spos.p;
  p.range_loc = (const float *)g.range_loc.p;
  p.items = (PPItem *)g.items.p;
  p.sched = (int32_t *)g.sched.p;
  p.item_cap = item_cap;
  p.vp = d.vp;
  p.mass2 = mass * mass;
  p.kick = kick;
  p.out = (float *)g.out.p;
  p.want_vmax = 1;
  p.err = ctr + 2;
  p.num_sms = g.num_sms;
  p.pairs = pairs;
  p.shape = 0;
  if (!pairs) CK(choose_pp_shape(m, d.n_used, p, st));
  launch_pp_items(p, st);
  g.launches += 3;
  CU(cudaGetLastError());
  if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][6], st));
  return CUBE_OK;
}

// PP force kernel on the compute stream, after run_pp_prep's work and the vp upload
static int run_pp_force(const PPArgs &p) {
  CK(wait_vp());
  if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][3], g.stream));
  launch_pp_force(p, g.stream);
  g.launches += 1;
  CU(cudaGetLastError());
  if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][4], g.stream));
  return CUBE_OK;
}

// PP force kernel group by group (consecutive tiles) for a host kick.  The launches alternate
// between the side streams (one launch's tail overlaps the next one's start); a group's launch
// waits for the binning and for that group's PM3 gather, and its vp range (its stored
// particles, a contiguous run of the spine) goes to the host on the copy stream as soon as the
// launch is done.  The compute stream ends after the last copy.
static int run_pp_force_tiles(const PPArgs &p, const Dev &d) {
  const Lay &L = g.L;
  if (!g.ready_tiles) {  // PM3 gathered all tiles at once
    CK(wait_vp());
    CU(cudaEventRecord(g.ev_pm3done, g.stream));
  }
  CU(cudaStreamWaitEvent(g.side2, g.ev_join, 0));  // binning (on side) done
  if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][3], g.side));
  const int64_t rows = (int64_t)L.nte * L.nte;
  for (int kk = 0; kk < g.ngrp; kk++) {
    const int k = g.grp_order[kk];
    cudaStream_t st = (kk & 1) ? g.side2 : g.side;
    CU(cudaStreamWaitEvent(st, g.ready_tiles ? g.ev_ready[k] : g.ev_pm3done, 0));
    launch_pp_force(p, st, g.grp_lo[k], g.grp_lo[k + 1]);
    g.launches += 1;
    CU(cudaGetLastError());
    CU(cudaEventRecord(g.ev_tile[k], st));
  }
  // copies after all launches: a copy into pageable host memory returns only when done
  for (int kk = 0; kk < g.ngrp; kk++) {
    const int k = g.grp_order[kk];
    const int t0 = g.grp_lo[k], t1 = g.grp_lo[k + 1];
    const int64_t lo = t0 ? d.h_idx[t0 * rows - 1] : 0, hi = d.h_idx[t1 * rows - 1];
    if (hi <= lo) continue;
    CU(cudaStreamWaitEvent(g.copy, g.ev_tile[k], 0));
    CU(cudaMemcpyAsync(d.h_vp + 3 * lo, d.vp + 3 * lo, sizeof(float) * 3 * (hi - lo), cudaMemcpyDeviceToHost,
                       g.copy));
  }
  g.vp_copied = true;
  CU(cudaEventRecord(g.ev_join, g.side));
  CU(cudaEventRecord(g.ev_join2, g.side2));
  CU(cudaStreamWaitEvent(g.stream, g.ev_join, 0));
  CU(cudaStreamWaitEvent(g.stream, g.ev_join2, 0));
  if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][4], g.stream));
  CU(cudaEventRecord(g.ev_copied, g.copy));
  CU(cudaStreamWaitEvent(g.stream, g.ev_copied, 0));
  return CUBE_OK;
}

// PP stage on the compute stream alone
static int run_pp(const Meta &m, const Dev &d, float mass, float kick, size_t &soff,
                  unsigned long long *pairs = nullptr) {
  PPArgs p{};
  CK(run_pp_prep(m, d, mass, kick, soff, p, g.stream, pairs));
  return run_pp_force(p);
}

static bool configured() { return g.configured; }

// Whole device pipeline on device inputs; outputs land in g.out (+ err word).
static int run_kick(const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf, const float *apm3,
                    const float *const *gk, const Dev &d, float mass, float a_mid, float dt, bool do_pm3,
                    bool do_pp, Meta &m) {
  if (!configured()) return fail(CUBE_ERR_NOT_CONFIGURED);
  CK(build_meta(ires, ixyz3, ratio_sf, apm3, m));
  CK(stage_begin((size_t)4 << 20));
  CK(grow(g.cell_base, sizeof(int64_t) * (size_t)g.L.ntile * g.L.nte * g.L.nte * g.L.nte));
  CK(grow(g.out, sizeof(float) * 8));
  CK(grow(g.counters, sizeof(int32_t) * 128));
  size_t soff = 0;
  // kick coefficient a_mid*dt/6/pi (kick.f90:529, pp_force_kernel.c:355)
  const float kick = (float)((double)(a_mid * dt / 6.0f) / 3.14159265358979323846);
  CU(cudaMemsetAsync(g.out.p, 0, sizeof(float) * 8, g.stream));
  CU(cudaMemsetAsync(g.counters.p, 0, sizeof(int32_t) * 128, g.stream));
  if (g.timing) {
    g.ring_cur = g.ring_next;
    g.ring_next = (g.ring_next + 1) % Ctx::kRing;
    g.ring_count = std::min(g.ring_count + 1, Ctx::kRing);
    g.ring_pm3[g.ring_cur] = do_pm3;
    g.ring_pp[g.ring_cur] = do_pp;
    CU(cudaEventRecord(g.ring[g.ring_cur][0], g.stream));
  }
  launch_cell_table(g.L, d.rhoc, d.idx, (int64_t *)g.cell_base.p, g.stream);
  g.launches += 1;
  CU(cudaGetLastError());
  if (do_pm3 && do_pp) {
    // the PP binning needs only xp and the cell table: it runs beside PM3
    PPArgs pa{};
    CU(cudaEventRecord(g.ev_fork, g.stream));
    CU(cudaStreamWaitEvent(g.side, g.ev_fork, 0));
    CK(run_pp_prep(m, d, mass, kick, soff, pa, g.side, nullptr));
    CU(cudaEventRecord(g.ev_join, g.side));
    g.ready_tiles = false;
    CK(run_pm3(m, ires, ratio_sf, gk, d, mass, kick, false, soff));
    if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][1], g.stream));
    if (d.h_vp && g.ngrp > 0) {
      CK(run_pp_force_tiles(pa, d));
    } else {
      CU(cudaStreamWaitEvent(g.stream, g.ev_join, 0));
      CK(run_pp_force(pa));
    }
  } else {
    if (do_pm3) CK(run_pm3(m, ires, ratio_sf, gk, d, mass, kick, !do_pp, soff));
    if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][1], g.stream));
    if (do_pp) CK(run_pp(m, d, mass, kick, soff));
  }
  if (g.timing) CU(cudaEventRecord(g.ring[g.ring_cur][5], g.stream));
  CK(stage_end());
  // error word next to the outputs
  CU(cudaMemcpyAsync((char *)g.out.p + 5 * sizeof(float), (char *)g.counters.p + 2 * sizeof(int32_t),
                     sizeof(int32_t), cudaMemcpyDeviceToDevice, g.stream));
  return CUBE_OK;
}

static int finish_times(bool do_pm3, bool do_pp) {
  if (!g.timing) return CUBE_OK;
  CU(cudaEventSynchronize(g.ring[g.ring_cur][5]));
  float a = 0, b = 0, c = 0, t = 0;
  if (do_pm3) CU(cudaEventElapsedTime(&a, g.ring[g.ring_cur][0], g.ring[g.ring_cur][1]));
  if (do_pp) {
    CU(cudaEventElapsedTime(&b, g.ring[g.ring_cur][2], g.ring[g.ring_cur][6]));
    CU(cudaEventElapsedTime(&c, g.ring[g.ring_cur][3], g.ring[g.ring_cur][4]));
  }
  CU(cudaEventElapsedTime(&t, g.ring[g.ring_cur][0], g.ring[g.ring_cur][5]));
  g.stage_ms[0] = a;
  g.stage_ms[1] = b;
  g.stage_ms[2] = c;
  g.stage_ms[3] = t;
  return CUBE_OK;
}

static int check_err_word(int32_t w) {
  if (!w) return CUBE_OK;
  if (w & (1 << CUBE_ERR_CAPACITY)) return fail(CUBE_ERR_CAPACITY);
  if (w & (1 << CUBE_ERR_TIMEOUT)) return fail(CUBE_ERR_TIMEOUT);
  return fail(CUBE_ERR_INVALID);
}

// host-buffer kick: upload, run, download vp and the outputs
static int host_kick(const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf, const float *apm3,
                     const float *const *gk, const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp,
                     float *vp, float mass, float a_mid, float dt, bool do_pm3, bool do_pp, float out5[5],
                     Meta &m) {
  if (!configured()) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!rhoc || !idx_b_r || !xp || !vp) return fail(CUBE_ERR_INVALID);
  CK(build_meta(ires, ixyz3, ratio_sf, apm3, m));  // host-side validation before touching the device
  if (do_pp && !apm3) return fail(CUBE_ERR_INVALID);
  const Lay &L = g.L;
  const int64_t nrows = (int64_t)L.ntile * L.nte * L.nte;
  const int64_t n_used = idx_b_r[nrows - 1];  // pm3_fft_cuda.cu:533-536
  if (n_used < 0 || n_used >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  // The spine must be non-decreasing and consistent with the rhoc row sums.  The tile groups'
  // bounds are checked before the uploads (they size the copies); the full check runs on the
  // host while the copies are under way, and a failure returns before any kernel is launched,
  // with the caller's arrays untouched.
  const int64_t rows_per_tile = (int64_t)L.nte * L.nte;
  for (int t = 1; t <= L.ntile; t++) {
    const int64_t a = idx_b_r[(t - 1) * rows_per_tile], b = idx_b_r[t * rows_per_tile - 1];
    const int64_t before = t > 1 ? idx_b_r[(t - 1) * rows_per_tile - 1] : 0;
    if (a < before || b < a || b > n_used) return fail(CUBE_ERR_INVALID);
  }
  auto spine_ok = [&]() {
    int64_t prev = 0;
    for (int64_t r = 0; r < nrows; r++) {
      int64_t s = 0;
      for (int i = 0; i < L.nte; i++) {
        const int32_t c = rhoc[r * L.nte + i];
        if (c < 0) return false;
        s += c;
      }
      if (idx_b_r[r] - prev != s) return false;
      prev = idx_b_r[r];
    }
    return true;
  };
  if (const int dst = ensure_device(); dst != CUBE_OK)  // no device: still report a bad spine as such
    return spine_ok() ? dst : fail(CUBE_ERR_INVALID);
  CK(grow(g.xp, sizeof(int16_t) * 3 * (size_t)std::max<int64_t>(n_used, 1)));
  CK(grow(g.vp, sizeof(float) * 3 * (size_t)std::max<int64_t>(n_used, 1)));
  CK(grow(g.rhoc, sizeof(int32_t) * (size_t)nrows * L.nte));
  CK(grow(g.idx, sizeof(int64_t) * (size_t)nrows));
  CU(cudaMemcpyAsync(g.rhoc.p, rhoc, sizeof(int32_t) * nrows * L.nte, cudaMemcpyHostToDevice, g.stream));
  CU(cudaMemcpyAsync(g.idx.p, idx_b_r, sizeof(int64_t) * nrows, cudaMemcpyHostToDevice, g.stream));
  g.ngrp = 0;
  if (n_used) {
    // xp group by group, so that the deposit of the first tiles overlaps the copy of the rest
    // (the copy stream first waits for the compute stream's earlier work on these buffers)
    CU(cudaEventRecord(g.ev_fork, g.stream));
    CU(cudaStreamWaitEvent(g.copy, g.ev_fork, 0));
    const int64_t rows = (int64_t)L.nte * L.nte;
    // groups of consecutive tiles, at most kMaxTileEvents of them
    g.ngrp = std::min(L.ntile, Ctx::kPipeGroups);
    for (int k = 0; k <= g.ngrp; k++) g.grp_lo[k] = (int)((int64_t)k * L.ntile / g.ngrp);
    for (int k = 0; k < g.ngrp; k++) {
      const int t0 = g.grp_lo[k], t1 = g.grp_lo[k + 1];
      const int64_t lo = t0 ? idx_b_r[t0 * rows - 1] : 0, hi = idx_b_r[t1 * rows - 1];
      if (hi > lo)
        CU(cudaMemcpyAsync((int16_t *)g.xp.p + 3 * lo, xp + 3 * lo, sizeof(int16_t) * 3 * (hi - lo),
                           cudaMemcpyHostToDevice, g.copy));
      CU(cudaEventRecord(g.ev_xp[k], g.copy));
    }
    g.xp_pending = true;
    g.xp_tiles = g.ngrp;
    // The groups are gathered, kicked by PP and copied back largest first, so that the last
    // PP launch and the last copy, which nothing overlaps, are the shortest.
    {
      int64_t cnt[Ctx::kMaxTileEvents];
      for (int k = 0; k < g.ngrp; k++) {
        const int t0 = g.grp_lo[k], t1 = g.grp_lo[k + 1];
        cnt[k] = idx_b_r[t1 * rows - 1] - (t0 ? idx_b_r[t0 * rows - 1] : 0);
        g.grp_order[k] = k;
      }
      std::stable_sort(g.grp_order, g.grp_order + g.ngrp, [&](int x, int y) { return cnt[x] > cnt[y]; });
    }
    // vp travels beside the deposit and FFTs, group by group in that order; its users wait for
    // their part
    for (int kk = 0; kk < g.ngrp; kk++) {
      const int k = g.grp_order[kk];
      const int t0 = g.grp_lo[k], t1 = g.grp_lo[k + 1];
      const int64_t lo = t0 ? idx_b_r[t0 * rows - 1] : 0, hi = idx_b_r[t1 * rows - 1];
      if (hi > lo)
        CU(cudaMemcpyAsync((float *)g.vp.p + 3 * lo, vp + 3 * lo, sizeof(float) * 3 * (hi - lo),
                           cudaMemcpyHostToDevice, g.copy));
      CU(cudaEventRecord(g.ev_vp[k], g.copy));
    }
    g.vp_tiles = g.ngrp;
    g.vp_pending = true;
  }
  if (!spine_ok()) {  // nothing launched yet: let the uploads finish and return
    cudaStreamSynchronize(g.copy);
    cudaStreamSynchronize(g.stream);
    g.xp_pending = g.vp_pending = false;
    g.xp_tiles = g.vp_tiles = 0;
    return fail(CUBE_ERR_INVALID);
  }
  Dev d{(const int16_t *)g.xp.p, (const int32_t *)g.rhoc.p, (const int64_t *)g.idx.p, (float *)g.vp.p, n_used};
  d.h_vp = vp;
  d.h_idx = idx_b_r;
  g.vp_copied = false;
  const int st = run_kick(ires, ixyz3, ratio_sf, apm3, gk, d, mass, a_mid, dt, do_pm3, do_pp, m);
  // also on a failed run: later work on these buffers must follow the uploads
  const int xst = wait_xp(g.stream);
  g.xp_pending = false;
  const int wst = xst != CUBE_OK ? xst : wait_vp();
  if (st != CUBE_OK || wst != CUBE_OK) {
    cudaStreamSynchronize(g.copy);
    cudaStreamSynchronize(g.side);
    cudaStreamSynchronize(g.side2);
    cudaStreamSynchronize(g.stream);
    return st != CUBE_OK ? st : wst;
  }
  if (n_used && !g.vp_copied)
    CU(cudaMemcpyAsync(vp, g.vp.p, sizeof(float) * 3 * n_used, cudaMemcpyDeviceToHost, g.stream));
  CU(cudaMemcpyAsync(g.h_out, g.out.p, sizeof(float) * 6, cudaMemcpyDeviceToHost, g.stream));
  CU(cudaStreamSynchronize(g.stream));
  CK(finish_times(do_pm3, do_pp));
  int32_t w;
  memcpy(&w, &g.h_out[5], sizeof(w));
  CK(check_err_word(w));
  for (int q = 0; q < 5; q++) out5[q] = g.h_out[q];
  return CUBE_OK;
}

}  // namespace cube

using namespace cube;

extern "C" {

int cube_set_layout(const cube_layout *l) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!l) return fail(CUBE_ERR_INVALID);
  const int rcs = l->ratio_cs;
  if (l->ng <= 0 || l->nnt <= 0 || l->nns <= 0 || rcs <= 0 || l->ngb <= 0) return fail(CUBE_ERR_INVALID);
  if (l->ng % rcs || (l->ng / rcs) % l->nnt || ((l->ng / rcs) / l->nnt) % l->nns) return fail(CUBE_ERR_INVALID);
  if (l->ngb % rcs || l->ngb < rcs) return fail(CUBE_ERR_INVALID);
  if (l->p_order != 2) return fail(CUBE_ERR_INVALID);
  if (l->pm3_mode != CUBE_PM3_SUBTILE && l->pm3_mode != CUBE_PM3_PERIODIC && l->pm3_mode != CUBE_PM3_TILE_PERIODIC)
    return fail(CUBE_ERR_INVALID);
  if (!(l->app >= 0.f)) return fail(CUBE_ERR_INVALID);
  Lay L{};
  L.ng = l->ng;
  L.nnt = l->nnt;
  L.nns = l->nns;
  L.rcs = rcs;
  L.ngb = l->ngb;
  L.nc = L.ng / rcs;
  L.nt = L.nc / L.nnt;
  L.ntt = L.nt / L.nns;
  L.ncb = L.ngb / rcs;
  L.nte = L.nt + 2 * L.ncb;
  L.ns3 = (L.nnt * L.nns) * (L.nnt * L.nns) * (L.nnt * L.nns);
  L.ntile = L.nnt * L.nnt * L.nnt;
  L.app = l->app;
  L.pm3_mode = l->pm3_mode;
  L.apm3f = l->apm3f;
  L.apm_range = l->apm_range;
  L.p_order = l->p_order;
  g.L = L;
  g.pub = *l;
  g.configured = true;
  t_last_error = CUBE_OK;
  return CUBE_OK;
}

int cube_pp_set_shape(int32_t shape) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (shape < -1 || shape >= pp_num_shapes()) return fail(CUBE_ERR_INVALID);
  g.pp_fixed = shape;
  if (shape < 0) g.pp_tuned.clear();
  return CUBE_OK;
}

int cube_pp_shapes(cube_pp_shape_info *out, int32_t cap, int32_t *n_shapes, int32_t *current) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (cap < 0 || (cap > 0 && !out)) return fail(CUBE_ERR_INVALID);
  const int ns = pp_num_shapes();
  if (n_shapes) *n_shapes = ns;
  if (current) *current = g.pp_last;
  for (int k = 0; k < std::min<int>(cap, ns); k++) {
    const PPShapeDesc d = pp_shape_desc(k);
    out[k].chunk = d.chunk;
    out[k].jtile = d.jtile;
    out[k].unroll = d.unroll;
    out[k].blocks = d.blocks;
    out[k].packed = d.packed;
    out[k].ms = g.pp_ms[k];
  }
  return CUBE_OK;
}

int cube_pp_work_stats(int64_t out[4]) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out) return fail(CUBE_ERR_INVALID);
  for (int k = 0; k < 4; k++) out[k] = 0;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!g.items.p || !g.sched.p) return CUBE_OK;  // no PP kick yet
  CU(cudaDeviceSynchronize());
  int32_t n = 0;
  CU(cudaMemcpy(&n, (const int32_t *)g.sched.p + sched_total_index(g.L.ntile), sizeof(int32_t),
                cudaMemcpyDeviceToHost));
  const size_t cap = g.items.cap / sizeof(PPItem);
  if (n < 0 || (size_t)n > cap) return fail(CUBE_ERR_CAPACITY);
  std::vector<PPItem> it((size_t)n);
  if (n) CU(cudaMemcpy(it.data(), g.items.p, sizeof(PPItem) * (size_t)n, cudaMemcpyDeviceToHost));
  std::unordered_map<uint32_t, int> per_cell;
  for (const PPItem &x : it) per_cell[x.cell]++;
  for (const PPItem &x : it) {
    const int ni = x.dims & 0xff, span = (x.dims >> 24) & 0xff;
    if (per_cell[x.cell] > 1) out[1]++;
    if (span > 0) out[2]++;
    out[3] = std::max<int64_t>(out[3], ni);
  }
  out[0] = n;
  return CUBE_OK;
}

int cube_get_layout(cube_layout *l) {
  if (!l) return fail(CUBE_ERR_INVALID);
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  *l = g.pub;
  return CUBE_OK;
}

int cube_last_error(void) { return t_last_error; }

const char *cube_error_string(int s) {
  switch (s) {
    case CUBE_OK: return "ok";
    case CUBE_ERR_INVALID: return "invalid argument or subtile metadata";
    case CUBE_ERR_NOT_CONFIGURED: return "cube_set_layout has not been called";
    case CUBE_ERR_CUDA: return "CUDA runtime error";
    case CUBE_ERR_CUFFT: return "cuFFT error";
    case CUBE_ERR_CAPACITY: return "device capacity check failed";
    case CUBE_ERR_NO_DEVICE: return "no CUDA device visible";
    case CUBE_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "unknown status";
  }
}

int cube_pm3_force(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf,
                   const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp, const float *const gk[5],
                   float *vp, float mass, float a_mid, float dt, float *f2max, float vmax[3], double *ptotal) {
  (void)isort;  // subtiles are independent; order only steered the reference's CPU scheduling
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  float out[5];
  Meta m;
  CK(host_kick(ires, ixyz3, ratio_sf, nullptr, gk, rhoc, idx_b_r, xp, vp, mass, a_mid, dt, true, false, out, m));
  if (f2max) *f2max = out[0];
  if (vmax) {
    vmax[0] = out[2];
    vmax[1] = out[3];
    vmax[2] = out[4];
  }
  if (ptotal) fill_ptotal(m, rhoc, ptotal);
  return CUBE_OK;
}

int cube_pp_force(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                  const int32_t *ratio_sf, const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp,
                  float *vp, float mass, float a_mid, float dt, float *f2max, float vmax[3], double *ptotal,
                  double *ttotal) {
  (void)isort;
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!apm3) return fail(CUBE_ERR_INVALID);
  const bool was = g.timing;
  g.timing = true;
  float out[5];
  Meta m;
  int s = host_kick(ires, ixyz3, ratio_sf, apm3, nullptr, rhoc, idx_b_r, xp, vp, mass, a_mid, dt, false, true, out,
                    m);
  g.timing = was;
  CK(s);
  if (f2max) *f2max = out[1];
  if (vmax) {
    vmax[0] = out[2];
    vmax[1] = out[3];
    vmax[2] = out[4];
  }
  if (ptotal) fill_ptotal(m, rhoc, ptotal);
  if (ttotal) {
    const Lay &L = g.L;
    for (int it = 0; it < L.ns3; it++) ttotal[it] = 0.0;
    const int nss = L.nns * L.nns * L.nns;
    const double sec = (g.stage_ms[1] + g.stage_ms[2]) * 1e-3 / L.ntile;
    for (int t = 0; t < L.ntile; t++) ttotal[m.owner[t * nss]] = sec;
  }
  return CUBE_OK;
}

int cube_kick_fine(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                   const int32_t *ratio_sf, const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp,
                   const float *const gk[5], float *vp, float mass, float a_mid, float dt, float out[5],
                   double *ptotal) {
  (void)isort;
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!apm3 || !out) return fail(CUBE_ERR_INVALID);
  Meta m;
  CK(host_kick(ires, ixyz3, ratio_sf, apm3, gk, rhoc, idx_b_r, xp, vp, mass, a_mid, dt, true, true, out, m));
  if (ptotal) fill_ptotal(m, rhoc, ptotal);
  return CUBE_OK;
}

int cube_kick_fine_device(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                          const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r,
                          const int16_t *d_xp, int64_t n_used, const float *const gk[5], float *d_vp, float mass,
                          float a_mid, float dt, float *d_out, void *stream) {
  (void)isort;
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  // an image without particles may pass null particle arrays
  if (!apm3 || !d_rhoc || !d_idx_b_r || !d_out || (n_used > 0 && (!d_xp || !d_vp))) return fail(CUBE_ERR_INVALID);
  if (n_used < 0 || n_used >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  cudaStream_t own = g.stream;
  if (stream) g.stream = (cudaStream_t)stream;
  Dev d{d_xp, d_rhoc, d_idx_b_r, d_vp, n_used};
  Meta m;
  int s = run_kick(ires, ixyz3, ratio_sf, apm3, gk, d, mass, a_mid, dt, true, true, m);
  if (s == CUBE_OK) {
    cudaError_t e = cudaMemcpyAsync(d_out, g.out.p, sizeof(float) * 6, cudaMemcpyDeviceToDevice, g.stream);
    if (e != cudaSuccess) s = fail(CUBE_ERR_CUDA);
  }
  g.stream = own;
  return s;
}

// ---- PM1 and PM2, the long-range layers (kick.f90:61-105, particle_mesh.f90, pm_thread) ----

// PM1: one periodic mesh of nc^3 coarse cells over the image (gridsize = ratio_cs, so the mesh
// coordinate is the global coarse coordinate), Green_3D(nc, apm_soft, 0, ratio_cs)
// (initialize.f90:129).  PM2: per parent tile the fine mesh of the tile with its buffers,
// ngt = (nt + 2 ncb) ratio_cs points per side (gridsize 1), all stored cells deposited
// (nloop = ncb), the physical ones kicked, Green_3D(ngt, apm_soft, apm_range, 1)
// (initialize.f90:135, kick.f90:82-88); the tiles' meshes go through one batched transform.
// Both kick vp of the physical particles by a_mid dt / (6 pi) times the TSC-gathered force.
static int run_pm_layer(int layer, const Dev &d, float mass, float kick, float apm_soft, float apm_range,
                        float out[5]) {
  const Lay &L = g.L;
  const bool pm1 = layer == 1;
  const int n = pm1 ? L.nc : L.nte * L.rcs;
  const int nslots = pm1 ? 1 : L.ntile;
  const int64_t n3 = (int64_t)n * n * n, nk = (int64_t)n * n * (n / 2 + 1);
  CK(stage_begin((size_t)1 << 20));
  CK(grow(g.cell_base, sizeof(int64_t) * (size_t)L.ntile * L.nte * L.nte * L.nte));
  CK(grow(g.out, sizeof(float) * 8));
  CK(grow(g.rho, sizeof(float) * n3 * nslots));
  CK(grow(g.rhok, sizeof(cufftComplex) * nk * nslots));
  CK(grow(g.force, sizeof(float) * n3 * 3 * nslots));
  float *G = nullptr;
  CK(get_green_params(n, apm_soft, pm1 ? 0.0f : apm_range, pm1 ? (float)L.rcs : 1.0f, &G));
  // mesh coordinate = stored coordinate * ratio_cs / gridsize (kick.f90:438, particle_mesh.f90:31)
  const double scale = pm1 ? 1.0 : (double)L.rcs;
  std::vector<MeshJob> jobs(L.ntile);
  for (int t = 0; t < L.ntile; t++) {
    const int tc[3] = {t % L.nnt, (t / L.nnt) % L.nnt, t / (L.nnt * L.nnt)};
    MeshJob &J = jobs[t];
    J.t = t;
    J.slot = pm1 ? 0 : t;
    J.range = 0.f;
    for (int q = 0; q < 3; q++) {
      J.lo[q] = pm1 ? L.ncb : 0;  // PM2 deposits the buffer cells too (nloop = ncb)
      J.alo[q] = L.ncb;
      J.off[q] = pm1 ? -(double)tc[q] * L.nt : 0.0;
    }
  }
  size_t soff = 0;
  CK(upload(g.jobs, jobs.data(), jobs.size(), soff));
  CU(cudaMemsetAsync(g.out.p, 0, sizeof(float) * 8, g.stream));
  launch_cell_table(L, d.rhoc, d.idx, (int64_t *)g.cell_base.p, g.stream);
  PM3Args a{};
  a.L = &g.L;
  a.rsf = 1;
  a.n = n;
  a.nslots = nslots;
  a.jobs = (const MeshJob *)g.jobs.p;
  a.njobs = L.ntile;
  for (int q = 0; q < 3; q++) {
    a.rdep[q] = pm1 ? L.nt : L.nte;
    a.ract[q] = L.nt;
  }
  a.wrap = pm1 ? 1 : 0;
  a.shift = pm1 ? 0 : L.ncb * L.rcs;  // array index = Fortran index - (1 - ngb)
  a.fphys_lo = pm1 ? 0 : L.ncb * L.rcs;
  a.fphys_n = pm1 ? n : L.nt * L.rcs;
  a.scale = scale;
  a.xp = d.xp;
  a.rhoc = d.rhoc;
  a.cell_base = (const int64_t *)g.cell_base.p;
  a.rho = (float *)g.rho.p;
  a.rhok = (cufftComplex *)g.rhok.p;
  a.force = (float *)g.force.p;
  a.green = G;
  a.mass = mass;
  a.kick = kick;
  a.vp = d.vp;
  a.out = (float *)g.out.p;
  a.want_vmax = 1;
  cufftHandle fw, bw;
  CK(get_plan(n, nslots, CUFFT_R2C, &fw));
  CK(get_plan(n, nslots, CUFFT_C2R, &bw));
  CU(cudaMemsetAsync(g.rho.p, 0, sizeof(float) * n3 * nslots, g.stream));
  launch_pm3_deposit(a, g.stream);
  CF(cufftExecR2C(fw, (cufftReal *)g.rho.p, (cufftComplex *)g.rhok.p));
  launch_pm3_kspace(a, g.stream);
  CF(cufftExecC2R(bw, (cufftComplex *)g.rhok.p, (cufftReal *)g.rho.p));
  launch_pm3_force(a, g.stream);
  launch_pm3_gather(a, g.stream);
  g.launches += 5;
  CU(cudaGetLastError());
  CK(stage_end());
  CU(cudaMemcpyAsync(out, g.out.p, sizeof(float) * 5, cudaMemcpyDeviceToHost, g.stream));
  CU(cudaStreamSynchronize(g.stream));
  return CUBE_OK;
}

static int pm_layer_entry(int layer, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp,
                          int64_t n_used, float *d_vp, float mass, float a_mid, float dt, float apm_soft,
                          float apm_range, float *f2max, float vmax[3], void *stream) {
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!d_rhoc || !d_idx_b_r || (n_used > 0 && (!d_xp || !d_vp)) || n_used < 0) return fail(CUBE_ERR_INVALID);
  if (!(apm_soft > 0.f) || apm_range < 0.f) return fail(CUBE_ERR_INVALID);
  const Lay &L = g.L;
  if (layer == 2 && L.pm3_mode == CUBE_PM3_TILE_PERIODIC) return fail(CUBE_ERR_INVALID);
  if (layer == 1 && (L.nc % 4 || L.nc < 8)) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  cudaStream_t own = g.stream;
  if (stream) g.stream = (cudaStream_t)stream;
  const float kick = (float)((double)(a_mid * dt / 6.0f) / 3.14159265358979323846);
  Dev d{d_xp, d_rhoc, d_idx_b_r, d_vp, n_used};
  float out[5] = {0, 0, 0, 0, 0};
  const int s = run_pm_layer(layer, d, mass, kick, apm_soft, apm_range, out);
  g.stream = own;
  if (s != CUBE_OK) return s;
  if (f2max) *f2max = out[0];
  if (vmax) {
    vmax[0] = out[2];
    vmax[1] = out[3];
    vmax[2] = out[4];
  }
  return CUBE_OK;
}

int cube_pm1_force_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                          float *d_vp, float mass, float a_mid, float dt, float apm1c, float *f2max, float vmax[3],
                          void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  return pm_layer_entry(1, d_rhoc, d_idx_b_r, d_xp, n_used, d_vp, mass, a_mid, dt, apm1c, 0.f, f2max, vmax,
                        stream);
}

int cube_pm2_force_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                          float *d_vp, float mass, float a_mid, float dt, float apm2, float apm1, float *f2max,
                          float vmax[3], void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  return pm_layer_entry(2, d_rhoc, d_idx_b_r, d_xp, n_used, d_vp, mass, a_mid, dt, apm2, apm1, f2max, vmax, stream);
}

// ---- drift and buffer rebuild ----

// drift.f90:26 in float: nlayer = 2 * ceiling(dt_mid * vz_max / ratio_cs) + 2
static int drift_nlayer(float dt_mid, float vz_max, int rcs, int *nlayer) {
  volatile float prod = dt_mid * vz_max;
  volatile float q = prod / (float)rcs;
  if (!std::isfinite(q) || q < 0.0f || q > 1.0e6f) return fail(CUBE_ERR_INVALID);
  *nlayer = 2 * (int)std::ceil(q) + 2;
  return CUBE_OK;
}

// One drift of the image plus the rebuild of its buffers, device arrays, on stream st.
static int drift_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, const float *d_vp,
                        const int64_t *d_pid, int64_t n_used, float dt_mid, float vz_max, int32_t *d_rhoc_new,
                        int64_t *d_idx_b_r_new, int16_t *d_xp_new, float *d_vp_new, int64_t *d_pid_new,
                        int64_t cap_new, int64_t *n_used_new, int64_t *n_physical, cudaStream_t st) {
  const Lay &L = g.L;
  if (!d_rhoc || !d_idx_b_r || !d_rhoc_new || !d_idx_b_r_new || !n_used_new) return fail(CUBE_ERR_INVALID);
  if (n_used < 0 || n_used >= ((int64_t)1 << 31) - 1 || cap_new < 0) return fail(CUBE_ERR_INVALID);
  if (n_used > 0 && (!d_xp || !d_vp)) return fail(CUBE_ERR_INVALID);
  if (cap_new > 0 && (!d_xp_new || !d_vp_new || (d_pid && !d_pid_new))) return fail(CUBE_ERR_INVALID);
  const int64_t ncs = (int64_t)L.ntile * L.nte * L.nte * L.nte;
  const int64_t ndest = (int64_t)L.nc * L.nc * L.nc;
  const int64_t nrows = (int64_t)L.ntile * L.nte * L.nte;
  if (ncs >= ((int64_t)1 << 31) || ndest >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  if (L.nt < L.ncb) return fail(CUBE_ERR_INVALID);  // a buffer mirrors at most one tile deep
  int nlayer = 0;
  CK(drift_nlayer(dt_mid, vz_max, L.rcs, &nlayer));
  const int64_t run_cap = std::max<int64_t>(n_used, 1) + drift_run_slack(g.num_sms);
  if (run_cap >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  CK(grow(g.dr_cb, sizeof(int64_t) * ncs));
  CK(grow(g.dr_cb_new, sizeof(int64_t) * ncs));
  CK(grow(g.dr_runrank, sizeof(uint32_t) * run_cap));
  CK(grow(g.dr_run_base, sizeof(int32_t) * ncs));
  CK(grow(g.dr_runs, drift_run_bytes() * run_cap));
  CK(grow(g.dr_ctr, sizeof(int32_t) * 8));
  CK(grow(g.dr_dest_runs, sizeof(int32_t) * ndest));
  CK(grow(g.dr_dest_start, sizeof(int32_t) * (ndest + 1)));
  CK(grow(g.dr_scan_tmp, sizeof(int32_t) * scan_tmp_elems(ndest)));
  CK(grow(g.dr_cursor, sizeof(int32_t) * ndest));
  CK(grow(g.dr_phys, sizeof(int32_t) * ndest));
  CK(grow(g.dr_list, sizeof(int32_t) * run_cap));
  CK(grow(g.dr_off, sizeof(int64_t) * run_cap));
  CK(grow(g.dr_rows, sizeof(int64_t) * nrows));
  CK(grow(g.dr_total, sizeof(int64_t) * 2));
  int32_t *ctr = (int32_t *)g.dr_ctr.p;
  CU(cudaMemsetAsync(ctr, 0, sizeof(int32_t) * 8, st));
  CU(cudaMemsetAsync(g.dr_dest_runs.p, 0, sizeof(int32_t) * ndest, st));
  CU(cudaMemsetAsync(g.dr_phys.p, 0, sizeof(int32_t) * ndest, st));
  CU(cudaMemsetAsync(g.dr_cursor.p, 0, sizeof(int32_t) * ndest, st));
  launch_cell_table(L, d_rhoc, d_idx_b_r, (int64_t *)g.dr_cb.p, st);
  DriftArgs a{};
  a.L = &g.L;
  a.nlayer = nlayer;
  a.dt_mid = dt_mid;
  a.num_sms = g.num_sms;
  a.n_used = n_used;
  a.rhoc = d_rhoc;
  a.cell_base = (const int64_t *)g.dr_cb.p;
  a.xp = d_xp;
  a.vp = d_vp;
  a.pid = d_pid;
  a.runrank = (uint32_t *)g.dr_runrank.p;
  a.run_base = (int32_t *)g.dr_run_base.p;
  a.runs = g.dr_runs.p;
  a.run_cap = (int32_t)run_cap;
  a.ctr = ctr;
  a.dest_runs = (int32_t *)g.dr_dest_runs.p;
  a.phys_count = (int32_t *)g.dr_phys.p;
  a.err = ctr + 4;
  a.dest_start = (int32_t *)g.dr_dest_start.p;
  a.cursor = (int32_t *)g.dr_cursor.p;
  a.run_list = (int32_t *)g.dr_list.p;
  a.run_off = (int64_t *)g.dr_off.p;
  a.rhoc_new = d_rhoc_new;
  a.cell_base_new = (const int64_t *)g.dr_cb_new.p;
  a.xp_new = d_xp_new;
  a.vp_new = d_vp_new;
  a.pid_new = d_pid ? d_pid_new : nullptr;
  launch_drift_runs(a, st);
  launch_drift_spine(a, d_rhoc_new, (int64_t *)g.dr_rows.p, d_idx_b_r_new, (int64_t *)g.dr_total.p, st);
  launch_cell_table(L, d_rhoc_new, d_idx_b_r_new, (int64_t *)g.dr_cb_new.p, st);
  g.launches += 6;
  CU(cudaGetLastError());
  // the new sizes decide whether the outputs fit: one host synchronisation
  int32_t h_ctr[8];
  int64_t h_total = 0;
  CU(cudaMemcpyAsync(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(&h_total, g.dr_total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  *n_used_new = h_total;
  if (n_physical) *n_physical = h_ctr[1];
  if (h_ctr[4] & (1 << CUBE_ERR_CAPACITY)) return fail(CUBE_ERR_CAPACITY);
  if (h_ctr[4]) return fail(CUBE_ERR_INVALID);
  if (h_total > cap_new || h_total >= ((int64_t)1 << 31)) return fail(CUBE_ERR_CAPACITY);
  a.n_used_new = h_total;
  launch_drift_place(a, h_ctr[0], (int32_t *)g.dr_scan_tmp.p, st);
  g.launches += 7;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(&h_ctr[4], ctr + 4, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (h_ctr[4]) return fail(CUBE_ERR_INVALID);
  return CUBE_OK;
}

int cube_drift_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, const float *d_vp,
                      const int64_t *d_pid, int64_t n_used, float dt_mid, float vz_max, int32_t *d_rhoc_new,
                      int64_t *d_idx_b_r_new, int16_t *d_xp_new, float *d_vp_new, int64_t *d_pid_new,
                      int64_t cap_new, int64_t *n_used_new, int64_t *n_physical, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  CK(ensure_device());
  return drift_device(d_rhoc, d_idx_b_r, d_xp, d_vp, d_pid, n_used, dt_mid, vz_max, d_rhoc_new, d_idx_b_r_new,
                      d_xp_new, d_vp_new, d_pid_new, cap_new, n_used_new, n_physical,
                      stream ? (cudaStream_t)stream : g.stream);
}

int cube_buffer_v_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, float *d_vp, int64_t n_used,
                         void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!d_rhoc || !d_idx_b_r || (n_used > 0 && !d_vp) || n_used < 0) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const Lay &L = g.L;
  cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
  CK(grow(g.dr_cb, sizeof(int64_t) * (size_t)L.ntile * L.nte * L.nte * L.nte));
  launch_cell_table(L, d_rhoc, d_idx_b_r, (int64_t *)g.dr_cb.p, st);
  launch_halo_velocities(L, d_rhoc, (const int64_t *)g.dr_cb.p, d_vp, n_used, g.num_sms, st);
  g.launches += 2;
  CU(cudaGetLastError());
  return CUBE_OK;
}

int cube_drift(int32_t *rhoc, int64_t *idx_b_r, int16_t *xp, float *vp, int64_t *pid, int64_t n_used,
               int64_t capacity, float dt_mid, float vz_max, int64_t *n_used_new, int64_t *n_physical) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!rhoc || !idx_b_r || !n_used_new || n_used < 0 || capacity < n_used) return fail(CUBE_ERR_INVALID);
  if (n_used > 0 && (!xp || !vp)) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const Lay &L = g.L;
  const size_t ncs = (size_t)L.ntile * L.nte * L.nte * L.nte, nrows = (size_t)L.ntile * L.nte * L.nte;
  const size_t nin = (size_t)std::max<int64_t>(n_used, 1), nout = (size_t)std::max<int64_t>(capacity, 1);
  CK(grow(g.dh_rhoc, sizeof(int32_t) * ncs));
  CK(grow(g.dh_idx, sizeof(int64_t) * nrows));
  CK(grow(g.dh_xp, sizeof(int16_t) * 3 * nin));
  CK(grow(g.dh_vp, sizeof(float) * 3 * nin));
  CK(grow(g.dh_rhoc2, sizeof(int32_t) * ncs));
  CK(grow(g.dh_idx2, sizeof(int64_t) * nrows));
  CK(grow(g.dh_xp2, sizeof(int16_t) * 3 * nout));
  CK(grow(g.dh_vp2, sizeof(float) * 3 * nout));
  if (pid) {
    CK(grow(g.dh_pid, sizeof(int64_t) * nin));
    CK(grow(g.dh_pid2, sizeof(int64_t) * nout));
  }
  cudaStream_t st = g.stream;
  CU(cudaMemcpyAsync(g.dh_rhoc.p, rhoc, sizeof(int32_t) * ncs, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(g.dh_idx.p, idx_b_r, sizeof(int64_t) * nrows, cudaMemcpyHostToDevice, st));
  if (n_used > 0) {
    CU(cudaMemcpyAsync(g.dh_xp.p, xp, sizeof(int16_t) * 3 * n_used, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(g.dh_vp.p, vp, sizeof(float) * 3 * n_used, cudaMemcpyHostToDevice, st));
    if (pid) CU(cudaMemcpyAsync(g.dh_pid.p, pid, sizeof(int64_t) * n_used, cudaMemcpyHostToDevice, st));
  }
  int64_t n_new = 0;
  const int s = drift_device((const int32_t *)g.dh_rhoc.p, (const int64_t *)g.dh_idx.p, (const int16_t *)g.dh_xp.p,
                             (const float *)g.dh_vp.p, pid ? (const int64_t *)g.dh_pid.p : nullptr, n_used, dt_mid,
                             vz_max, (int32_t *)g.dh_rhoc2.p, (int64_t *)g.dh_idx2.p, (int16_t *)g.dh_xp2.p,
                             (float *)g.dh_vp2.p, pid ? (int64_t *)g.dh_pid2.p : nullptr, capacity, &n_new,
                             n_physical, st);
  *n_used_new = n_new;
  if (s != CUBE_OK) return s;  // the host arrays are untouched
  CU(cudaMemcpyAsync(rhoc, g.dh_rhoc2.p, sizeof(int32_t) * ncs, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(idx_b_r, g.dh_idx2.p, sizeof(int64_t) * nrows, cudaMemcpyDeviceToHost, st));
  if (n_new > 0) {
    CU(cudaMemcpyAsync(xp, g.dh_xp2.p, sizeof(int16_t) * 3 * n_new, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(vp, g.dh_vp2.p, sizeof(float) * 3 * n_new, cudaMemcpyDeviceToHost, st));
    if (pid) CU(cudaMemcpyAsync(pid, g.dh_pid2.p, sizeof(int64_t) * n_new, cudaMemcpyDeviceToHost, st));
  }
  CU(cudaStreamSynchronize(st));
  return CUBE_OK;
}

// ---- checkpoint files ----

int cube_snapshot_write(const char *prefix, const char *suffix, const cube_sim_header *header, const int32_t *rhoc,
                        const int64_t *idx_b_r, const int16_t *xp, const float *vp, const int64_t *pid) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  const int s = snapshot_write(g.L, prefix, suffix, header, rhoc, idx_b_r, xp, vp, pid);
  return s == CUBE_OK ? s : fail(s);
}

int cube_snapshot_read(const char *prefix, const char *suffix, cube_sim_header *header, int32_t *rhoc_phys,
                       int16_t *xp, float *vp, int64_t *pid, int64_t capacity) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  const int s = snapshot_read(g.L, prefix, suffix, header, rhoc_phys, xp, vp, pid, capacity);
  return s == CUBE_OK ? s : fail(s);
}

// ---- CIC power spectrum (utilities/cicpower.f90, utilities/powerspectrum.f90) ----

int cube_kick_sums(const int32_t *d_rhoc, const int64_t *d_idx_b_r, int64_t n_used, const float *d_va,
                   const float *d_vb, float mass, double out[8], void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!d_rhoc || !d_idx_b_r || !out || n_used < 0 || (n_used > 0 && (!d_va || !d_vb))) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  CK(grow(g.ks_out, sizeof(double) * kNumKickSums));
  cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
  CU(cudaMemsetAsync(g.ks_out.p, 0, sizeof(double) * kNumKickSums, st));
  launch_kick_sums(g.L, d_rhoc, d_idx_b_r, d_va, d_vb, mass, (double *)g.ks_out.p, st);
  g.launches += 1;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(out, g.ks_out.p, sizeof(double) * kNumKickSums, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return CUBE_OK;
}

int cube_learned_fallback(const int32_t *d_rhoc, const int64_t *d_idx_b_r, int64_t n_used, const float *d_vp0,
                          const float *d_vp_learned, const float *d_vp_full, float bound, int32_t samples,
                          float *d_vp_out, double out[5], void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!d_rhoc || !d_idx_b_r || !out || n_used < 0 || samples < 1 || samples > 32 || !(bound >= 0.f))
    return fail(CUBE_ERR_INVALID);
  if (n_used > 0 && (!d_vp0 || !d_vp_learned || !d_vp_full || !d_vp_out)) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  CK(grow(g.fb_out, sizeof(double) * 8));
  cudaStream_t st = stream ? (cudaStream_t)stream : g.stream;
  unsigned long long *stats = (unsigned long long *)g.fb_out.p;
  double *err = (double *)g.fb_out.p + 4;
  CU(cudaMemsetAsync(g.fb_out.p, 0, sizeof(double) * 8, st));
  if (n_used > 0 && d_vp_out != d_vp_learned)
    CU(cudaMemcpyAsync(d_vp_out, d_vp_learned, sizeof(float) * 3 * (size_t)n_used, cudaMemcpyDeviceToDevice, st));
  launch_learned_fallback(g.L, d_rhoc, d_idx_b_r, d_vp0, d_vp_learned, d_vp_full, bound, samples, d_vp_out, stats,
                          err, st);
  g.launches += 1;
  CU(cudaGetLastError());
  unsigned long long hs[4];
  double he[2];
  CU(cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(he, err, sizeof(he), cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  out[0] = (double)hs[0];
  out[1] = (double)hs[1];
  out[2] = (double)hs[2];
  out[3] = he[1] > 0.0 ? std::sqrt(he[0] / he[1]) : 0.0;
  out[4] = (double)samples;
  return CUBE_OK;
}

int cube_power_spectrum(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                        int64_t n_physical, int32_t nw, int32_t nbin, double *bins, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!d_rhoc || !d_idx_b_r || !bins || (n_used > 0 && !d_xp) || n_physical <= 0) return fail(CUBE_ERR_INVALID);
  if (nw < 2 || nw > 2048 || (nw & 1)) return fail(CUBE_ERR_INVALID);
  if (nbin <= 0) nbin = (int)std::lround((nw / 2) * std::sqrt(3.0));
  if (nbin > 4096) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const Lay &L = g.L;
  const int64_t n3 = (int64_t)nw * nw * nw, nk = (int64_t)nw * nw * (nw / 2 + 1);
  CK(grow(g.dr_cb, sizeof(int64_t) * (size_t)L.ntile * L.nte * L.nte * L.nte));
  CK(grow(g.pw_grid, sizeof(float) * n3));
  CK(grow(g.pw_k, sizeof(cufftComplex) * nk));
  CK(grow(g.pw_bins, sizeof(double) * 4 * (nbin + 1)));
  cudaStream_t own = g.stream;
  if (stream) g.stream = (cudaStream_t)stream;
  cudaStream_t st = g.stream;
  int s = CUBE_OK;
  do {
    if (cudaMemsetAsync(g.pw_grid.p, 0, sizeof(float) * n3, st) != cudaSuccess ||
        cudaMemsetAsync(g.pw_bins.p, 0, sizeof(double) * 4 * (nbin + 1), st) != cudaSuccess) {
      s = fail(CUBE_ERR_CUDA);
      break;
    }
    launch_cell_table(L, d_rhoc, d_idx_b_r, (int64_t *)g.dr_cb.p, st);
    launch_cic_grid(L, nw, d_rhoc, (const int64_t *)g.dr_cb.p, d_xp, n_used, (float *)g.pw_grid.p, g.num_sms, st);
    launch_density_contrast((float *)g.pw_grid.p, n3, (float)((double)n3 / (double)n_physical), st);
    cufftHandle fw;
    s = get_plan(nw, 1, CUFFT_R2C, &fw);
    if (s != CUBE_OK) break;
    if (cufftExecR2C(fw, (cufftReal *)g.pw_grid.p, (cufftComplex *)g.pw_k.p) != CUFFT_SUCCESS) {
      s = fail(CUBE_ERR_CUFFT);
      break;
    }
    launch_pk_bins((const cufftComplex *)g.pw_k.p, nw, nbin, (double *)g.pw_bins.p, g.num_sms, st);
    g.launches += 4;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(bins, g.pw_bins.p, sizeof(double) * 4 * (nbin + 1), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      s = fail(CUBE_ERR_CUDA);
  } while (0);
  g.stream = own;
  return s;
}

// ---- learned PP shell ----

struct cube_mlp {
  cube::MlpParams p;
};

static void mlp_free(cube_mlp *h) {
  MlpParams &p = h->p;
  void *bufs[] = {p.master, p.grad, p.mom, p.vel, p.wb, p.wt, p.xb, p.a[0], p.a[1], p.a[2], p.dyb, p.dzb, p.dzt,
                  p.at, p.tb, p.z[0], p.z[1], p.z[2], p.y, p.dy, p.dz, p.da, p.b4pad, p.err};
  for (void *b : bufs)
    if (b) cudaFree(b);
  delete h;
}

int cube_mlp_create(const float *params, int32_t batch_cap, cube_mlp **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!params || !out || batch_cap <= 0 || batch_cap % 16) return fail(CUBE_ERR_INVALID);
  *out = nullptr;
  CK(ensure_device());
  cube_mlp *h = new cube_mlp;
  MlpParams &p = h->p;
  p.device = g.device;
  p.cap = batch_cap;
  const size_t B = (size_t)batch_cap, W = kMlpW;
  bool ok = true;
  auto al = [&](auto **ptr, size_t bytes) {
    if (ok && cudaMalloc((void **)ptr, bytes) != cudaSuccess) ok = false;
  };
  al(&p.master, sizeof(float) * kMlpParams);
  al(&p.grad, sizeof(float) * kMlpParams);
  al(&p.mom, sizeof(float) * kMlpParams);
  al(&p.vel, sizeof(float) * kMlpParams);
  al(&p.wb, sizeof(__nv_bfloat16) * kMlpWbElems);
  al(&p.wt, sizeof(__nv_bfloat16) * kMlpWbElems);
  al(&p.xb, sizeof(__nv_bfloat16) * B * kMlpK1);
  for (int l = 0; l < 3; l++) {
    al(&p.a[l], sizeof(__nv_bfloat16) * B * W);
    al(&p.z[l], sizeof(float) * B * W);
  }
  al(&p.dyb, sizeof(__nv_bfloat16) * B * kMlpOutPad);
  al(&p.dzb, sizeof(__nv_bfloat16) * B * W);
  al(&p.dzt, sizeof(__nv_bfloat16) * B * W);
  al(&p.at, sizeof(__nv_bfloat16) * B * W);
  al(&p.tb, sizeof(float) * B * kMlpOut);
  al(&p.y, sizeof(float) * B * kMlpOutPad);
  al(&p.dy, sizeof(float) * B * kMlpOutPad);
  al(&p.dz, sizeof(float) * B * W);
  al(&p.da, sizeof(float) * B * W);
  al(&p.b4pad, sizeof(float) * kMlpOutPad);
  al(&p.err, sizeof(int32_t));
  if (ok) ok = cudaMemset(p.err, 0, sizeof(int32_t)) == cudaSuccess;
  if (ok) ok = cudaMemcpy(p.master, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok) ok = cudaMemset(p.mom, 0, sizeof(float) * kMlpParams) == cudaSuccess &&
               cudaMemset(p.vel, 0, sizeof(float) * kMlpParams) == cudaSuccess &&
               cudaMemset(p.grad, 0, sizeof(float) * kMlpParams) == cudaSuccess;
  if (ok) {
    launch_mlp_pack(p, g.stream);
    ok = cudaStreamSynchronize(g.stream) == cudaSuccess;
  }
  if (!ok) {
    mlp_free(h);
    return fail(CUBE_ERR_CUDA);
  }
  *out = h;
  return CUBE_OK;
}

int cube_mlp_destroy(cube_mlp *h) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!h) return CUBE_OK;
  cudaSetDevice(h->p.device);
  cudaDeviceSynchronize();
  mlp_free(h);
  return CUBE_OK;
}

int cube_mlp_get_params(cube_mlp *h, float *params, float *grads) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!h || (!params && !grads)) return fail(CUBE_ERR_INVALID);
  CU(cudaSetDevice(h->p.device));
  CU(cudaDeviceSynchronize());
  if (params) CU(cudaMemcpy(params, h->p.master, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  if (grads) CU(cudaMemcpy(grads, h->p.grad, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
  return CUBE_OK;
}

// positions of the stored copies and the fine-grid density of the image, on stream s
static int mlp_prepare(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                       cudaStream_t s) {
  const Lay &L = g.L;
  if (L.pm3_mode != CUBE_PM3_PERIODIC) return fail(CUBE_ERR_INVALID);  // one periodic image
  CK(grow(g.cell_base, sizeof(int64_t) * (size_t)L.ntile * L.nte * L.nte * L.nte));
  CK(grow(g.mlp_pos, sizeof(float4) * (size_t)std::max<int64_t>(n_used, 1)));
  CK(grow(g.mlp_rho, sizeof(float) * (size_t)L.ng * L.ng * L.ng));
  launch_cell_table(L, d_rhoc, d_idx_b_r, (int64_t *)g.cell_base.p, s);
  launch_mlp_pos(L, d_xp, d_rhoc, (const int64_t *)g.cell_base.p, (float4 *)g.mlp_pos.p, s);
  launch_mlp_density((const float4 *)g.mlp_pos.p, n_used, L.ng, (float *)g.mlp_rho.p, s);
  g.launches += 3;
  CU(cudaGetLastError());
  return CUBE_OK;
}

int cube_mlp_features(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                      void *d_X, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!d_rhoc || !d_idx_b_r || !d_xp || !d_X || n_used < 0) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  cudaStream_t s = stream ? (cudaStream_t)stream : g.stream;
  CK(mlp_prepare(d_rhoc, d_idx_b_r, d_xp, n_used, s));
  launch_mlp_features((const float4 *)g.mlp_pos.p, n_used, (const float *)g.mlp_rho.p, g.L.ng,
                      (__nv_bfloat16 *)d_X, s);
  g.launches += 1;
  CU(cudaGetLastError());
  return CUBE_OK;
}

int cube_mlp_train_step(cube_mlp *h, const void *d_X, const float *d_T, const int32_t *d_rows, int32_t batch,
                        float lr, float *d_loss, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!h || !d_X || !d_T || !d_rows || !d_loss) return fail(CUBE_ERR_INVALID);
  CU(cudaSetDevice(h->p.device));
  const int st = mlp_train_step(h->p, (const __nv_bfloat16 *)d_X, d_T, d_rows, batch, lr, d_loss,
                                stream ? (cudaStream_t)stream : g.stream);
  return st == CUBE_OK ? CUBE_OK : fail(st);
}

int cube_mlp_forward(cube_mlp *h, const void *d_X, int64_t rows, float *d_Y, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!h || !d_X || !d_Y || rows < 0) return fail(CUBE_ERR_INVALID);
  CU(cudaSetDevice(h->p.device));
  const int st = mlp_forward(h->p, (const __nv_bfloat16 *)d_X, rows, d_Y, stream ? (cudaStream_t)stream : g.stream);
  return st == CUBE_OK ? CUBE_OK : fail(st);
}

int cube_mlp_kick(cube_mlp *h, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp,
                  int64_t n_used, float *d_vp, float scale, float a_mid, float dt, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!h || !d_rhoc || !d_idx_b_r || !d_xp || !d_vp || n_used < 0) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  cudaStream_t s = stream ? (cudaStream_t)stream : g.stream;
  CK(mlp_prepare(d_rhoc, d_idx_b_r, d_xp, n_used, s));
  // the kick coefficient of run_kick (kick.f90:529), times the network's output scale
  const float kick = (float)((double)(a_mid * dt / 6.0f) / 3.14159265358979323846);
  launch_mlp_apply(h->p, (const float4 *)g.mlp_pos.p, (const float *)g.mlp_rho.p, g.L.ng, n_used, d_vp,
                   kick * scale, g.num_sms, s);
  g.launches += 1;
  CU(cudaGetLastError());
  // the inference kernel's bounded waits report through a status word: read it once the kick is done
  int32_t e = 0;
  CU(cudaMemcpyAsync(&e, h->p.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (e) return fail(CUBE_ERR_TIMEOUT);
  return CUBE_OK;
}

// A captured kick: the graph, its executable form, the pinned staging area its table uploads
// read from, and the number of library kernels one replay launches.
struct cube_kick_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *stage = nullptr;
  int device = -1;
  long long launches = 0;
};

int cube_kick_graph_create(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                           const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r,
                           const int16_t *d_xp, int64_t n_used, float *d_vp, float mass, float a_mid, float dt,
                           float *d_out, cube_kick_graph **out) {
  (void)isort;
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!out) return fail(CUBE_ERR_INVALID);
  *out = nullptr;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  // the subtile geometry synchronises the host between mesh batches, which a graph cannot hold
  if (g.L.pm3_mode == CUBE_PM3_SUBTILE) return fail(CUBE_ERR_INVALID);
  if (!apm3 || !d_rhoc || !d_idx_b_r || !d_out || (n_used > 0 && (!d_xp || !d_vp))) return fail(CUBE_ERR_INVALID);
  if (n_used < 0 || n_used >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const float *gk[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // 1. a kick on a scratch copy of vp sizes every buffer, plan and table outside the capture
  {
    float *scratch = nullptr;
    CU(cudaMalloc(&scratch, sizeof(float) * 3 * (size_t)std::max<int64_t>(n_used, 1)));
    cudaError_t e = n_used > 0 ? cudaMemcpyAsync(scratch, d_vp, sizeof(float) * 3 * n_used,
                                                 cudaMemcpyDeviceToDevice, g.stream)
                               : cudaSuccess;
    Meta m;
    Dev d{d_xp, d_rhoc, d_idx_b_r, scratch, n_used};
    int st = e == cudaSuccess ? run_kick(ires, ixyz3, ratio_sf, apm3, gk, d, mass, a_mid, dt, true, true, m)
                              : fail(CUBE_ERR_CUDA);
    cudaStreamSynchronize(g.stream);
    cudaFree(scratch);
    if (st != CUBE_OK) return st;
  }
  // 2. the capture, with the graph's own staging area and without the timing events
  cube_kick_graph *kg = new cube_kick_graph;
  kg->device = g.device;
  const size_t stage_bytes = (size_t)4 << 20;
  if (cudaMallocHost(&kg->stage, stage_bytes) != cudaSuccess) {
    delete kg;
    return fail(CUBE_ERR_CUDA);
  }
  const bool timing = g.timing;
  g.timing = false;
  g.stage_override = kg->stage;
  g.stage_override_cap = stage_bytes;
  const long long l0 = g.launches;
  int st = CUBE_OK;
  if (cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    st = fail(CUBE_ERR_CUDA);
  } else {
    Meta m;
    Dev d{d_xp, d_rhoc, d_idx_b_r, d_vp, n_used};
    st = run_kick(ires, ixyz3, ratio_sf, apm3, gk, d, mass, a_mid, dt, true, true, m);
    if (st == CUBE_OK &&
        cudaMemcpyAsync(d_out, g.out.p, sizeof(float) * 6, cudaMemcpyDeviceToDevice, g.stream) != cudaSuccess)
      st = fail(CUBE_ERR_CUDA);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(g.stream, &graph);  // always ends the capture
    kg->graph = graph;
    if (st == CUBE_OK && (e != cudaSuccess || !graph)) st = fail(CUBE_ERR_CUDA);
  }
  g.stage_override = nullptr;
  g.stage_override_cap = 0;
  g.timing = timing;
  kg->launches = g.launches - l0;
  g.launches = l0;
  if (st == CUBE_OK && cudaGraphInstantiate(&kg->exec, kg->graph, 0) != cudaSuccess) st = fail(CUBE_ERR_CUDA);
  if (st != CUBE_OK) {
    cudaGetLastError();  // a failed capture leaves its error behind
    if (kg->graph) cudaGraphDestroy(kg->graph);
    cudaFreeHost(kg->stage);
    delete kg;
    return st;
  }
  *out = kg;
  return CUBE_OK;
}

int cube_kick_graph_launch(cube_kick_graph *kg, void *stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!kg || !kg->exec) return fail(CUBE_ERR_INVALID);
  CU(cudaSetDevice(kg->device));
  CU(cudaGraphLaunch(kg->exec, (cudaStream_t)stream));
  g.launches += kg->launches;
  return CUBE_OK;
}

int cube_kick_graph_destroy(cube_kick_graph *kg) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!kg) return CUBE_OK;
  cudaSetDevice(kg->device);
  if (kg->exec) cudaGraphExecDestroy(kg->exec);
  if (kg->graph) cudaGraphDestroy(kg->graph);
  cudaStreamSynchronize(nullptr);
  if (kg->stage) cudaFreeHost(kg->stage);
  delete kg;
  return CUBE_OK;
}

void c_pm3_force_kernel(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf,
                        int32_t *rhoc, int64_t *idx_b_r, int16_t *xp, const float *g2, const float *g4,
                        const float *g6, const float *g8, const float *g12, float *vp, float mass, float a_mid,
                        float dt, float *f2max, float vmax[3], double *ptotal) {
  const float *gk[5] = {g2, g4, g6, g8, g12};
  cube_pm3_force(isort, ires, ixyz3, ratio_sf, rhoc, idx_b_r, xp, gk, vp, mass, a_mid, dt, f2max, vmax, ptotal);
}

void c_pp_force_kernel(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                       const int32_t *ratio_sf, int32_t *rhoc, int64_t *idx_b_r, int16_t *xp, float *vp,
                       float mass, float a_mid, float dt, float *f2max, float vmax[3], double *ptotal,
                       double *ttotal) {
  cube_pp_force(isort, ires, ixyz3, apm3, ratio_sf, rhoc, idx_b_r, xp, vp, mass, a_mid, dt, f2max, vmax, ptotal,
                ttotal);
}

void c_pm3_fft_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g.device < 0) return;
  cudaSetDevice(g.device);
  cudaStreamSynchronize(g.stream);
  for (auto &p : g.plans) cufftDestroy(p.h);
  g.plans.clear();
  for (auto &e : g.greens) cudaFree(e.d);
  g.greens.clear();
  for (auto &e : g.hgreens) cudaFree(e.d);
  g.hgreens.clear();
  release(g.rho);
  release(g.rhok);
  release(g.force);
  release(g.phi_pad);
  release(g.brick_ctr);
  release(g.dep_items);
  release(g.jobs);
  release(g.mlp_pos);
  release(g.mlp_rho);
}

void c_gpu_velocity_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g.device < 0) return;
  cudaSetDevice(g.device);
  cudaStreamSynchronize(g.stream);
  Buf *bufs[] = {&g.xp, &g.rhoc, &g.idx, &g.vp, &g.cell_base, &g.tiles, &g.count, &g.cell_start, &g.scan_tmp,
                 &g.spos, &g.spill, &g.spill_rank, &g.counters, &g.items, &g.range_loc, &g.sched, &g.out, &g.ks_out, &g.fb_out};
  for (Buf *b : bufs) release(*b);
}

int cube_pp_bin_tile(const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf, const int32_t *rhoc,
                     const int64_t *idx_b_r, const int16_t *xp, int32_t tile, int32_t spatial, uint32_t *keys,
                     int64_t *ip, int32_t *cell_start, float *xf, int64_t cap_n, int64_t cap_grid, int64_t *n_out,
                     int64_t *grid_out) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!rhoc || !idx_b_r || !xp) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const Lay &L = g.L;
  if (tile < 0 || tile >= L.ntile) return fail(CUBE_ERR_INVALID);
  Meta m;
  CK(build_meta(ires, ixyz3, ratio_sf, nullptr, m));
  const int64_t nrows = (int64_t)L.ntile * L.nte * L.nte;
  const int64_t n_used = idx_b_r[nrows - 1];
  if (n_used < 0 || n_used >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  CK(stage_begin((size_t)4 << 20));
  CK(grow(g.xp, sizeof(int16_t) * 3 * (size_t)std::max<int64_t>(n_used, 1)));
  CK(grow(g.rhoc, sizeof(int32_t) * (size_t)nrows * L.nte));
  CK(grow(g.idx, sizeof(int64_t) * (size_t)nrows));
  CK(grow(g.cell_base, sizeof(int64_t) * (size_t)nrows * L.nte));
  CK(grow(g.counters, sizeof(int32_t) * 128));
  CU(cudaMemcpyAsync(g.rhoc.p, rhoc, sizeof(int32_t) * nrows * L.nte, cudaMemcpyHostToDevice, g.stream));
  CU(cudaMemcpyAsync(g.idx.p, idx_b_r, sizeof(int64_t) * nrows, cudaMemcpyHostToDevice, g.stream));
  if (n_used)
    CU(cudaMemcpyAsync(g.xp.p, xp, sizeof(int16_t) * 3 * n_used, cudaMemcpyHostToDevice, g.stream));
  CU(cudaMemsetAsync(g.counters.p, 0, sizeof(int32_t) * 128, g.stream));
  launch_cell_table(L, (const int32_t *)g.rhoc.p, (const int64_t *)g.idx.p, (int64_t *)g.cell_base.p, g.stream);
  size_t soff = 0;
  CK(upload(g.tiles, m.tiles.data(), m.tiles.size(), soff));
  CK(grow(g.count, sizeof(int32_t) * (size_t)m.ncells));
  CK(grow(g.cell_start, sizeof(int32_t) * (size_t)(m.ncells + 1)));
  CK(grow(g.scan_tmp, sizeof(int32_t) * scan_tmp_elems(m.ncells)));
  CK(grow(g.spos, sizeof(float4) * (size_t)std::max<int64_t>(n_used, 1)));
  CK(grow(g.spill, sizeof(Spill) * 2048));
  CK(grow(g.spill_rank, sizeof(int32_t) * 2048));
  int32_t *ctr = (int32_t *)g.counters.p;
  BinArgs b{};
  b.L = &g.L;
  b.d_tiles = (const TilePP *)g.tiles.p;
  b.max_rcp = m.max_rcp;
  b.ncells = m.ncells;
  b.xp = (const int16_t *)g.xp.p;
  b.rhoc = (const int32_t *)g.rhoc.p;
  b.cell_base = (const int64_t *)g.cell_base.p;
  b.count = (int32_t *)g.count.p;
  b.cell_start = (int32_t *)g.cell_start.p;
  b.spos = (float4 *)g.spos.p;
  b.spill = (Spill *)g.spill.p;
  b.spill_rank = (int32_t *)g.spill_rank.p;
  b.spill_n = ctr;
  b.spill_cap = 2048;
  b.scan_tmp = (int32_t *)g.scan_tmp.p;
  b.err = ctr + 2;
  b.spatial = spatial ? 1 : 0;
  if (bin_smem_bytes(m.max_rcp) > 200 * 1024) return fail(CUBE_ERR_INVALID);
  launch_pp_binning(b, g.stream);
  CU(cudaGetLastError());
  CK(stage_end());
  const TilePP tp = m.tiles[tile];
  const int64_t grid = (int64_t)tp.S * tp.S * tp.S;
  std::vector<int32_t> cs(grid + 1);
  CU(cudaMemcpyAsync(cs.data(), (int32_t *)g.cell_start.p + tp.cell0, sizeof(int32_t) * (grid + 1),
                     cudaMemcpyDeviceToHost, g.stream));
  int32_t err = 0;
  CU(cudaMemcpyAsync(&err, ctr + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, g.stream));
  CU(cudaStreamSynchronize(g.stream));
  CK(check_err_word(err));
  const int32_t first = cs[0];
  const int64_t N = cs[grid] - first;
  if (n_out) *n_out = N;
  if (grid_out) *grid_out = grid;
  if (N > cap_n || grid + 1 > cap_grid) return fail(CUBE_ERR_CAPACITY);
  std::vector<float4> sp(N > 0 ? N : 1);
  if (N) CU(cudaMemcpy(sp.data(), (float4 *)g.spos.p + first, sizeof(float4) * N, cudaMemcpyDeviceToHost));
  if (cell_start)
    for (int64_t c = 0; c <= grid; c++) cell_start[c] = cs[c] - first;
  if (keys) {
    int64_t c = 0;
    for (int64_t q = 0; q < N; q++) {
      while (cs[c + 1] - first <= q) c++;
      keys[q] = (uint32_t)c;
    }
  }
  for (int64_t q = 0; q < N; q++) {
    if (ip) {
      int32_t v;
      memcpy(&v, &sp[q].w, sizeof(v));
      ip[q] = v;
    }
    if (xf) {
      xf[q] = sp[q].x;
      xf[N + q] = sp[q].y;
      xf[2 * N + q] = sp[q].z;
    }
  }
  return CUBE_OK;
}

int cube_pp_force_noalloc(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                          const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r,
                          const int16_t *d_xp, int64_t n_used, float *d_vp, float mass, float a_mid, float dt,
                          float *d_out, void *stream) {
  (void)isort;
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  // no context set-up here: the current device and the caller's stream are used as they are
  const int s = pp_force_noalloc(g.L, ires, ixyz3, apm3, ratio_sf, d_rhoc, d_idx_b_r, d_xp, n_used, d_vp, mass,
                                 a_mid, dt, d_out, (cudaStream_t)stream);
  if (s != CUBE_OK) return fail(s);
  return CUBE_OK;
}

int cube_pp_pair_count(const int32_t *ires, const int32_t *ixyz3, const float *apm3, const int32_t *ratio_sf,
                       const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp, int64_t *pairs) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!g.configured) return fail(CUBE_ERR_NOT_CONFIGURED);
  if (!rhoc || !idx_b_r || !xp || !apm3 || !pairs) return fail(CUBE_ERR_INVALID);
  Meta m;
  CK(build_meta(ires, ixyz3, ratio_sf, apm3, m));
  CK(ensure_device());
  const Lay &L = g.L;
  const int64_t nrows = (int64_t)L.ntile * L.nte * L.nte;
  const int64_t n_used = idx_b_r[nrows - 1];
  if (n_used < 0 || n_used >= ((int64_t)1 << 31)) return fail(CUBE_ERR_INVALID);
  CK(stage_begin((size_t)4 << 20));
  CK(grow(g.xp, sizeof(int16_t) * 3 * (size_t)std::max<int64_t>(n_used, 1)));
  CK(grow(g.rhoc, sizeof(int32_t) * (size_t)nrows * L.nte));
  CK(grow(g.idx, sizeof(int64_t) * (size_t)nrows));
  CK(grow(g.cell_base, sizeof(int64_t) * (size_t)nrows * L.nte));
  CK(grow(g.counters, sizeof(int32_t) * 128));
  CK(grow(g.out, sizeof(float) * 8));
  CU(cudaMemcpyAsync(g.rhoc.p, rhoc, sizeof(int32_t) * nrows * L.nte, cudaMemcpyHostToDevice, g.stream));
  CU(cudaMemcpyAsync(g.idx.p, idx_b_r, sizeof(int64_t) * nrows, cudaMemcpyHostToDevice, g.stream));
  if (n_used) CU(cudaMemcpyAsync(g.xp.p, xp, sizeof(int16_t) * 3 * n_used, cudaMemcpyHostToDevice, g.stream));
  CU(cudaMemsetAsync(g.counters.p, 0, sizeof(int32_t) * 128, g.stream));
  CU(cudaMemsetAsync(g.out.p, 0, sizeof(float) * 8, g.stream));
  launch_cell_table(L, (const int32_t *)g.rhoc.p, (const int64_t *)g.idx.p, (int64_t *)g.cell_base.p, g.stream);
  Dev d{(const int16_t *)g.xp.p, (const int32_t *)g.rhoc.p, (const int64_t *)g.idx.p, nullptr, n_used};
  size_t soff = 0;
  unsigned long long *d_pairs = (unsigned long long *)((int32_t *)g.counters.p + 8);
  CK(run_pp(m, d, 1.0f, 0.0f, soff, d_pairs));
  CK(stage_end());
  unsigned long long h = 0;
  int32_t err = 0;
  CU(cudaMemcpyAsync(&h, d_pairs, sizeof(h), cudaMemcpyDeviceToHost, g.stream));
  CU(cudaMemcpyAsync(&err, (int32_t *)g.counters.p + 2, sizeof(err), cudaMemcpyDeviceToHost, g.stream));
  CU(cudaStreamSynchronize(g.stream));
  CK(check_err_word(err));
  *pairs = (int64_t)h;
  return CUBE_OK;
}

int cube_green_table(int32_t n, float apm_soft, float apm_range, float gridsize, float *G) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (n < 2 || !G) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const size_t count = (size_t)n * n * (n / 2 + 1);
  float *d = nullptr;
  CU(cudaMalloc(&d, sizeof(float) * count));
  launch_green_fp64(n, apm_soft, apm_range, gridsize, 2, d, g.stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(G, d, sizeof(float) * count, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(CUBE_ERR_CUDA);
  return CUBE_OK;
}

int cube_force_truth_fp64(const double *pos, int64_t n, double box, double app, const int64_t *targets, int64_t nt,
                          double alpha, double rcut, int32_t nmax, double *F) {
  std::lock_guard<std::mutex> lk(g_mu);
  t_last_error = CUBE_OK;
  if (!pos || !targets || !F || n <= 0 || nt < 0 || box <= 0 || rcut > 0.5 * box) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  const int s = ewald_device(pos, n, box, app, targets, nt, alpha, rcut, nmax, F);
  if (s != CUBE_OK) return fail(s);
  return CUBE_OK;
}

int cube_stage_times(float ms[4]) {
  if (!ms) return fail(CUBE_ERR_INVALID);
  for (int q = 0; q < 4; q++) ms[q] = g.stage_ms[q];
  return CUBE_OK;
}

int cube_timing_read(float *ms, int32_t max_calls, int32_t *n_calls) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!ms || !n_calls || max_calls < 0) return fail(CUBE_ERR_INVALID);
  const int n = std::min(g.ring_count, (int)max_calls);
  const int first = (g.ring_next - g.ring_count + Ctx::kRing) % Ctx::kRing;
  for (int q = 0; q < n; q++) {
    const int s = (first + q) % Ctx::kRing;
    cudaEvent_t *e = g.ring[s];
    CU(cudaEventSynchronize(e[5]));
    float a = 0, b = 0, c = 0, t = 0;
    if (g.ring_pm3[s]) CU(cudaEventElapsedTime(&a, e[0], e[1]));
    if (g.ring_pp[s]) {
      CU(cudaEventElapsedTime(&b, e[2], e[6]));
      CU(cudaEventElapsedTime(&c, e[3], e[4]));
    }
    CU(cudaEventElapsedTime(&t, e[0], e[5]));
    ms[4 * q] = a;
    ms[4 * q + 1] = b;
    ms[4 * q + 2] = c;
    ms[4 * q + 3] = t;
  }
  *n_calls = n;
  g.ring_count = 0;
  return CUBE_OK;
}

int64_t cube_launch_count(void) { return g.launches; }

int cube_fp32_peak_probe(float *tflops) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!tflops) return fail(CUBE_ERR_INVALID);
  CK(ensure_device());
  float ms = 0.f;
  double flops = 0.0;
  if (fma_probe(g.stream, g.num_sms, &ms, &flops) != cudaSuccess) return fail(CUBE_ERR_CUDA);
  *tflops = (float)(flops / (ms * 1e-3) / 1e12);
  return CUBE_OK;
}

int cube_enable_timing(int on) {
  g.timing = on != 0;
  return CUBE_OK;
}

}  // extern "C"
