// Internal declarations shared by the kernels and the C-ABI layer.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include "../../include/cube2_b200.h"

namespace cube {

// Run-time layout; the derived sizes mirror parameters.f90:56-78.
struct Lay {
  int ng, nnt, nns, rcs, ngb;
  int nc, nt, ntt, ncb, nte, ns3, ntile;
  float app;
  int pm3_mode;
  float apm3f, apm_range;
  int p_order;
};

// Per-parent-tile PP grid (one fine-grid launch per tile, pp_force_kernel.cu:643-661).
struct TilePP {
  int rcp;         // PP cells per coarse cell (max ratio_sf over the tile's subtiles)
  int S;           // PP cells per side of the tile region (nt + 2 coarse cells) = rcp*(nt+2)
  int64_t cell0;   // first global PP cell index of this tile
};

// Spilled particle: its PP key lies in a neighbouring coarse cell because the
// reference's float rounding (pp_force_kernel.c:213-236) pushed it across.
struct Spill {
  int64_t gkey;  // global PP cell
  int32_t ip;    // storage index
  int32_t cell;  // t * R^3 + (cz*R + cy)*R + cx, region-local coarse cell
};

// PM3 mesh job (a periodic image tile, or one buffered subtile).
struct MeshJob {
  int t;          // parent tile
  int lo[3];      // first deposit coarse cell (C index into the extended tile)
  int alo[3];     // first active (gathered) coarse cell
  double off[3];  // mesh coordinate = (c - ncb + frac) * scale - off
  int slot;       // batch slot
  float range;    // unused by PM3 (kept for alignment of the table)
};

constexpr int kWarps = 8;  // warps per block in warp-per-cell kernels
constexpr int kPPChunk = 16;  // i-particles per PP work item of the default shape (a crowded PP cell is split into chunks)

// PP force kernel shape (pp.cu): i-particles per work item, staged candidates per warp, pair-loop
// unroll, resident blocks per SM the registers are budgeted for, pair law on packed f32x2
// arithmetic (two candidates per lane and instruction) or on scalar FP32
struct PPShapeDesc {
  int chunk, jtile, unroll, blocks, packed;
};
constexpr int kMaxPPShapes = 32;

// ---------------------------------------------------------------------------------------------
// device helpers

// Fixed-point decode of pp_force_kernel.c:213-218 / kick.f90:292 in double:
// (c) + (u + 0.5) * 2^-16 with u = (uint16)xp; exact.
__device__ __forceinline__ double decode_pos(int c, int16_t xp) {
  return (double)c + ((double)(uint16_t)xp + 0.5) * (1.0 / 65536.0);
}

__device__ __forceinline__ void atomic_max_nonneg(float *addr, float v) {
  // non-negative floats order like their bit patterns
  atomicMax(reinterpret_cast<int *>(addr), __float_as_int(v));
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ int64_t wrapi(int64_t a, int64_t n) {
  a %= n;
  return a < 0 ? a + n : a;
}

// ---------------------------------------------------------------------------------------------
// kernel launchers (defined in the .cu files); all enqueue on `s`

// cell_base[t][k][j][i] = idx_b_r[t][k][j] - sum(rhoc[t][k][j][i:])  (pp_force_kernel.c:203-209)
void launch_cell_table(const Lay &L, const int32_t *rhoc, const int64_t *idx_b_r, int64_t *cell_base,
                       cudaStream_t s);

// PP binning (counting sort by PP cell, bit-exact with pp_force_kernel.c:196-274)
struct BinArgs {
  const Lay *L;
  const TilePP *d_tiles;  // device table [ntile]
  int max_rcp;
  int64_t ncells;         // total PP cells over all tiles
  const int16_t *xp;
  const int32_t *rhoc;
  const int64_t *cell_base;
  int32_t *count;         // [ncells]
  int32_t *cell_start;    // [ncells + 1]
  float4 *spos;           // [n_region] x,y,z (fine units, tile-local), w = ip bits
  Spill *spill;           // [spill_cap]
  int32_t *spill_rank;    // [spill_cap]
  int32_t *spill_n;       // device counter
  int spill_cap;
  int32_t *scan_tmp;      // scan scratch
  int32_t *err;           // device error word
  int spatial;            // 1: order inside each PP cell by Morton sub-cell (kick); 0: reference order
};
void launch_pp_binning(const BinArgs &a, cudaStream_t s);
// No particle can spill into the next coarse cell's PP cells (exact float keys); then the
// binning can run tile by tile, each tile's launches right after its own xp arrives.
bool pp_binning_spill_free(const Lay &L, const TilePP *h_tiles);
// count, scan and place the PP regions of tiles [t_lo, t_hi); the tiles must be binned in order
// on one stream
void launch_pp_binning_tiles(const BinArgs &a, const TilePP *h_tiles, int t_lo, int t_hi, cudaStream_t s);
size_t bin_smem_bytes(int max_rcp);
size_t scan_tmp_elems(int64_t n);

// PP work list + force
// One PP work item (pp.cu): a chunk of at most `chunk` particles of one interior PP cell, with
// what its warp needs up front; k_pp_items fills it once per kick
struct __align__(16) PPItem {
  uint32_t cell;  // global PP cell index
  int32_t i0;     // first particle of the chunk in the cell-sorted order
  int32_t dims;   // ni | rcp << 8 | R << 16 | span << 24: particles, PP cells per coarse cell,
                  // stencil radius, 1 when the item holds two cells along x (x and x + 1)
  float rc;       // PP range of the cell
  float cep, k35, h, rc2;  // 2 / rc, 1 / (35 rc^2), ratio_cs / rcp, rc^2
};

struct PPArgs {
  const Lay *L;
  const TilePP *d_tiles;
  const TilePP *h_tiles;
  int64_t ncells;
  const int32_t *cell_start;
  const float4 *spos;
  const float *range_loc;   // [ns3] PP range by subtile location
  PPItem *items;            // [item_cap]
  int32_t *sched;           // [sched_ints(ntile)], zeroed by launch_pp_items: bucket counts and
                            // cursors per tile, tile bases, work-queue heads
  int64_t item_cap;
  float *vp;                // device vp [n_used][3]
  float mass2, kick;
  float *out;               // [5] f2max_pm3, f2max_pp, vmax[3]
  int want_vmax;
  int32_t *err;
  int num_sms;
  unsigned long long *pairs;  // non-null: count accepted pairs instead of kicking
  int shape;                  // kernel shape index (pp_shape_desc); 0 with `pairs`
};
// FP64 conservation sums of a kick over the physical particles (sums.cu): [0..2] sum m dv,
// [3] kinetic-energy change, [4..6] sum |m dv|, [7] particles; d_out is accumulated into
constexpr int kNumKickSums = 8;
void launch_kick_sums(const Lay &L, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const float *d_va,
                      const float *d_vb, float mass, double *d_out, cudaStream_t s);
// learned shell: per-cell check of the learned velocities against the full-cutoff ones on the
// first `samples` physical particles of each coarse cell; cells over the bound take the
// full-cutoff velocities (fallback.cu).  d_out must already hold a copy of d_vpl.
void launch_learned_fallback(const Lay &L, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const float *d_vp0,
                             const float *d_vpl, const float *d_vpf, float bound, int samples, float *d_out,
                             unsigned long long *d_stats, double *d_err, cudaStream_t s);
size_t sched_ints(int ntile);
int64_t sched_total_index(int ntile);  // where the work list's item count lies in `sched`
int pp_num_shapes();
PPShapeDesc pp_shape_desc(int i);
int pp_min_chunk();  // smallest chunk of any shape: the work list capacity is sized for it
// work list for the shape a.shape (shape 0 with a.pairs)
void launch_pp_items(const PPArgs &a, cudaStream_t s);
// force kernel over the items of tiles [t_lo, t_hi) (t_hi < 0: all tiles); disjoint tile ranges
// and the full range have their own queue heads, so launches over disjoint ranges may run on
// several streams
void launch_pp_force(const PPArgs &a, cudaStream_t s, int t_lo = 0, int t_hi = -1);

// PM3
struct PM3Args {
  const Lay *L;
  int rsf;
  int n;                 // mesh side
  int nslots;            // batch size
  const MeshJob *jobs;   // device [njobs]
  int njobs;
  int rdep[3], ract[3];  // deposit / active coarse ranges per job
  int wrap;              // 1 periodic image mesh, 0 buffered subtile mesh
  int shift;             // array index = floor(coord) + shift (nfb in buffered mode)
  int fphys_lo, fphys_n; // f2max region per slot (buffered mode)
  double scale;          // ratio_cs / gridsize
  const int16_t *xp;
  const int32_t *rhoc;
  const int64_t *cell_base;
  float *rho;            // [nslots][n^3] density, then potential
  cufftComplex *rhok;    // [nslots][n*n*(n/2+1)]
  float *force;          // [nslots*3][n^3]
  const float *green;    // [n*n*(n/2+1)]
  float mass, kick;
  float *vp;
  float *out;
  int want_vmax;
  int32_t *err = nullptr;  // device status word (bit CUBE_ERR_TIMEOUT from a bounded wait), may be null
  int num_sms = 148;
  float *phi_pad = nullptr;  // the potential with kPotPad ghost points per side (periodic images), [nslots][(n+2P)^3]
  int32_t *brick_ctr = nullptr;  // work counter of the brick kernels (one int, zeroed by the launcher)
  int2 *dep_items = nullptr;      // deposit work list: pm3_dep_items_bytes(...) of scratch
  int64_t n_particles_hint = 0;   // stored particles (sizes the deposit work list)
};
// scratch of the deposit work list for a launch over `njobs` jobs of `cells` coarse cells each
size_t pm3_dep_items_bytes(int64_t cells_per_job, int njobs, int64_t n_used);
constexpr int kPotPad = 4;  // ghost points per side of the padded potential of the brick kernels
int launch_pm3_deposit(const PM3Args &a, cudaStream_t s);  // returns the kernels it launched
void launch_pm3_kspace(const PM3Args &a, cudaStream_t s);
// the k-space step on the spectrum of two-dimensional x-y transforms: z transform, Green
// multiply, inverse z transform (mesh sides where pm3_kspace_z_ok)
bool pm3_kspace_z_ok(int n);
void launch_pm3_kspace_z(const PM3Args &a, cudaStream_t s);
void launch_pm3_force(const PM3Args &a, cudaStream_t s);  // force arrays + f2max from the potential
void launch_pm3_gather(const PM3Args &a, cudaStream_t s);
// periodic meshes: the force difference fused into the gather, brick by brick (no force arrays);
// returns false (nothing launched) where the brick geometry does not apply
int pm3_brick_mc(const PM3Args &a);
bool launch_pm3_force_gather(const PM3Args &a, cudaStream_t s);  // reads a.phi_pad
void launch_pm3_ghosts(const PM3Args &a, cudaStream_t s);          // fills the ghost points of a.phi_pad
void launch_green_fp64(int n, double apm_soft, double apm_range, double gridsize, int p_order, float *G,
                       cudaStream_t s);

// exclusive scan of int32 counts (binning.cu): out[i] = base + sum of in[0..i) for i <= n (base:
// a device int, or 0 when null), so out[n] = base + total; tmp has scan_tmp_elems(n) entries
void scan_exclusive_i32(const int32_t *in, int64_t n, int32_t *out, int32_t *tmp, cudaStream_t s,
                        const int32_t *base = nullptr);

// Drift of one image and the rebuild of its buffers (drift.cu)
struct DriftArgs {
  const Lay *L;
  int nlayer;            // drift.f90:26
  float dt_mid;
  int64_t n_used, n_used_new;  // stored copies of the current image and of the new one
  int num_sms;
  const int32_t *rhoc;   // current image
  const int64_t *cell_base;
  const int16_t *xp;
  const float *vp;
  const int64_t *pid;    // may be null
  uint32_t *runrank;     // [n_used]
  int32_t *run_base;     // [ntile * nte^3]
  void *runs;            // [run_cap] records of drift_run_bytes()
  int32_t run_cap;
  int32_t *ctr;          // [2] zeroed: runs, kept particles
  int32_t *dest_runs;    // [nc^3] zeroed
  int32_t *phys_count;   // [nc^3] zeroed
  int32_t *err;
  int32_t *dest_start;   // [nc^3 + 1]
  int32_t *cursor;       // [nc^3] zeroed
  int32_t *run_list;     // [run_cap]
  int64_t *run_off;      // [run_cap]
  const int32_t *rhoc_new;   // new image (spine from launch_drift_spine)
  const int64_t *cell_base_new;
  int16_t *xp_new;
  float *vp_new;
  int64_t *pid_new;
};
size_t drift_run_bytes();
// run-table slots beyond one per stored copy: the per-warp chunks' unused ends
int64_t drift_run_slack(int num_sms);
void launch_drift_runs(const DriftArgs &a, cudaStream_t s);
// new counts of every extended cell, row sums and the spine; *total = stored copies
void launch_drift_spine(const DriftArgs &a, int32_t *rhoc_new, int64_t *rows, int64_t *idx_b_r_new,
                        int64_t *total, cudaStream_t s);
void launch_drift_place(const DriftArgs &a, int32_t nruns, int32_t *scan_tmp, cudaStream_t s);
// buffer_v: every buffer copy takes the velocity of the physical particle it mirrors
void launch_halo_velocities(const Lay &L, const int32_t *rhoc, const int64_t *cell_base, float *vp, int64_t n_used,
                            int num_sms, cudaStream_t s);

// CIC power spectrum (power.cu): deposit of the physical particles on an nw^3 grid, density
// contrast, and the binning of the R2C transform into [4][nbin + 1] doubles (modes, sum |k|,
// sum |delta_k|^2 / sinc^4, sum 4 pi k^3 |delta_k|^2 / sinc^4)
void launch_cic_grid(const Lay &L, int nw, const int32_t *rhoc, const int64_t *cell_base, const int16_t *xp,
                     int64_t n_used, float *grid, int num_sms, cudaStream_t s);
void launch_density_contrast(float *grid, int64_t n, float scale, cudaStream_t s);
size_t pk_bins_smem(int nbin);
void launch_pk_bins(const cufftComplex *ck, int nw, int nbin, double *bins, int num_sms, cudaStream_t s);

// checkpoint files (snapshot.cu)
constexpr size_t kSimHeaderBytes = 13 * 8 + 19 * 4;
int snapshot_write(const Lay &L, const char *prefix, const char *suffix, const cube_sim_header *h,
                   const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp, const float *vp,
                   const int64_t *pid);
int snapshot_read(const Lay &L, const char *prefix, const char *suffix, cube_sim_header *h, int32_t *rhoc_phys,
                  int16_t *xp, float *vp, int64_t *pid, int64_t capacity);

// PP kick with all scratch in a static device array (noalloc.cu)
int pp_force_noalloc(const Lay &L, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                     const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp,
                     int64_t n_used, float *d_vp, float mass, float a_mid, float dt, float *d_out, cudaStream_t s);
size_t noalloc_scratch_bytes();

// Learned PP shell (mlp.cu).  FP32 master parameters, flat:
// W1 [128][80] b1 [128] W2 [128][128] b2 [128] W3 [128][128] b3 [128] W4 [3][128] b4 [3].
// BF16 copies per layer l: wb [Np][K] and their transposes wt [K][Np] (W4 padded to 16 rows).
constexpr int kMlpIn = 67, kMlpK1 = 80, kMlpW = 128, kMlpOut = 3, kMlpOutPad = 16;
__host__ __device__ constexpr int mlp_K(int l) { return l == 0 ? kMlpK1 : kMlpW; }
__host__ __device__ constexpr int mlp_N(int l) { return l == 3 ? kMlpOut : kMlpW; }
__host__ __device__ constexpr int mlp_Np(int l) { return l == 3 ? kMlpOutPad : kMlpW; }
__host__ __device__ constexpr int mlp_woff(int l) {
  return l == 0 ? 0 : mlp_woff(l - 1) + mlp_N(l - 1) * mlp_K(l - 1) + mlp_N(l - 1);
}
__host__ __device__ constexpr int mlp_boff(int l) { return mlp_woff(l) + mlp_N(l) * mlp_K(l); }
__host__ __device__ constexpr int mlp_wboff(int l) { return l == 0 ? 0 : mlp_wboff(l - 1) + mlp_Np(l - 1) * mlp_K(l - 1); }
constexpr int kMlpParams = mlp_boff(3) + kMlpOut;
constexpr int kMlpWbElems = mlp_wboff(3) + kMlpOutPad * kMlpW;

struct MlpParams {
  float *master = nullptr, *grad = nullptr, *mom = nullptr, *vel = nullptr;  // [kMlpParams]
  __nv_bfloat16 *wb = nullptr, *wt = nullptr;                                // [kMlpWbElems]
  int step = 0;
  int cap = 0;  // training batch capacity (rows)
  // training scratch for cap rows
  __nv_bfloat16 *xb = nullptr, *a[3] = {}, *dyb = nullptr, *dzb = nullptr, *dzt = nullptr, *at = nullptr;
  float *tb = nullptr, *z[3] = {}, *y = nullptr, *dy = nullptr, *dz = nullptr, *da = nullptr, *b4pad = nullptr;
  int device = -1;
  int32_t *err = nullptr;  // device status word of the inference kernel (bit CUBE_ERR_TIMEOUT)
};
void launch_mlp_pos(const Lay &L, const int16_t *xp, const int32_t *rhoc, const int64_t *cell_base, float4 *pos,
                    cudaStream_t s);
void launch_mlp_density(const float4 *pos, int64_t n, int ng, float *rho, cudaStream_t s);
void launch_mlp_features(const float4 *pos, int64_t n, const float *rho, int ng, __nv_bfloat16 *X, cudaStream_t s);
void launch_mlp_apply(const MlpParams &m, const float4 *pos, const float *rho, int ng, int64_t n, float *vp,
                      float coef, int num_sms, cudaStream_t s);
void launch_mlp_pack(MlpParams &m, cudaStream_t s);
int mlp_train_step(MlpParams &m, const __nv_bfloat16 *X, const float *T, const int32_t *rows, int batch, float lr,
                   float *loss, cudaStream_t s);
int mlp_forward(MlpParams &m, const __nv_bfloat16 *X, int64_t nrows, float *Y, cudaStream_t s);

// FP32 FMA throughput probe (5 launches); returns the time and the FLOPs executed
cudaError_t fma_probe(cudaStream_t s, int num_sms, float *ms, double *flops);

// FP64 truth
int ewald_device(const double *pos, int64_t n, double box, double app, const int64_t *targets, int64_t nt,
                 double alpha, double rcut, int nmax, double *F);

}  // namespace cube
