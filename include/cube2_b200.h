/*
 * cube2_b200 -- B200 (sm_100a) fine-scale kick of CUBE2: PM3 fine-mesh force
 * plus PP short-range pair force, behind the C ABI that CUBE2's Fortran
 * driver binds in kick.f90:12-46 and finalize.f90:8-13.
 *
 * Array conventions are the reference's (C views of Fortran arrays):
 *   xp       int16  [n_used][3]  fixed-point offset in the coarse cell
 *   vp       float  [n_used][3]
 *   rhoc     int32  [nnt][nnt][nnt][nte][nte][nte]   (tz,ty,tx,k,j,i; nte = nt + 2 ncb)
 *   idx_b_r  int64  [nnt][nnt][nnt][nte][nte]        running count at the end of row (j,k)
 *   ixyz3    int32  [ns3][6]   sx,sy,sz,tx,ty,tz (1-based), initialize.f90:207-224
 *   isort    int32  [ns3]      1-based, ires int32 [ns3] levels 2..6
 *   ratio_sf int32  [7],  apm3 float [7]
 * n_used = idx_b_r[last] (pm3_fft_cuda.cu:533-536).
 *
 * The reference fixes the layout at compile time (parameters.f90); this
 * library takes it at run time through cube_set_layout(), which the driver
 * calls once before the first kick.
 *
 * Errors never terminate the process.  The reference-named void entry points
 * record a status readable with cube_last_error(); the cube_* variants
 * return it.  A call rejected on the host (bad arguments, metadata or sizes)
 * leaves every output untouched.  A call whose failure is found on the
 * device (CUBE_ERR_CAPACITY or CUBE_ERR_INVALID from the device status word,
 * CUBE_ERR_TIMEOUT) has already run kernels: its outputs, vp included, are
 * then undefined (part of vp may hold the kick).
 */
#ifndef CUBE2_B200_H
#define CUBE2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cube_status {
  CUBE_OK = 0,
  CUBE_ERR_INVALID = 1,        /* bad argument or metadata (the reference aborts: pp_force_kernel.cu:985-986) */
  CUBE_ERR_NOT_CONFIGURED = 2, /* cube_set_layout() not called */
  CUBE_ERR_CUDA = 3,           /* CUDA runtime error */
  CUBE_ERR_CUFFT = 4,          /* cuFFT error */
  CUBE_ERR_CAPACITY = 5,       /* a device-side capacity check failed */
  CUBE_ERR_NO_DEVICE = 6,      /* no CUDA device visible */
  CUBE_ERR_TIMEOUT = 7         /* a bounded device wait gave up */
};

/* PM3 mesh geometry */
enum cube_pm3_mode {
  CUBE_PM3_SUBTILE = 0,       /* the reference's per-subtile buffered meshes, Green tables from the caller */
  CUBE_PM3_PERIODIC = 1,      /* one periodic mesh of side ng*ratio_sf over the image, Green table tabulated here */
  CUBE_PM3_TILE_PERIODIC = 2  /* every parent tile is its own periodic box (a batch of independent boxes whose
                                 buffers hold the tile's own periodic copies): one periodic mesh of side
                                 nt*ratio_cs*ratio_sf per tile, transformed as one batch */
};

typedef struct cube_layout {
  int32_t ng;       /* fine cells per image side          parameters.f90:20 */
  int32_t nnt;      /* tiles per image side               parameters.f90:24 */
  int32_t nns;      /* subtiles per tile side             parameters.f90:25 */
  int32_t ratio_cs; /* fine cells per coarse cell         parameters.f90:22 */
  int32_t ngb;      /* tile buffer in fine cells          parameters.f90:56 (ncb = ngb/ratio_cs) */
  float app;        /* PP softening in fine cells         parameters.f90:42 */
  int32_t pm3_mode; /* enum cube_pm3_mode */
  float apm3f;      /* PM3 softening in mesh cells, for the tabulated Green table (parameters.f90:38) */
  float apm_range;  /* PM3 range cut in mesh cells for the tabulated table, 0 = full force */
  int32_t p_order;  /* assignment order, 2 = TSC (parameters.f90:48); only 2 is supported */
} cube_layout;

/* Configure the layout (once, before the first kick).  Replaces the
 * compile-time constants of cuda_parameters_generated.h:4-14. */
int cube_set_layout(const cube_layout *layout);
int cube_get_layout(cube_layout *layout);

int cube_last_error(void);
const char *cube_error_string(int status);

/* ---- reference entry points (drop-in) ---- */

/* PM3 fine-mesh force and kick.  Replaces pm3_fft_cuda.cu:516-620 (bound at
 * kick.f90:31-45).  Unlike the reference CUDA build, vp is updated here (the
 * CPU path's semantics, kick.f90:529) instead of being parked in a device
 * accumulator that only the next c_pp_force_kernel call applies.  f2max,
 * vmax (max |vp| of the kicked particles) and ptotal (particles per subtile)
 * are written.  g2..g12 are the Green tables of levels 2..6 (mode
 * CUBE_PM3_SUBTILE; cached on the device keyed by pointer and size as
 * pm3_fft_cuda.cu:153-175 does); they are ignored in mode CUBE_PM3_PERIODIC. */
void c_pm3_force_kernel(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf,
                        int32_t *rhoc, int64_t *idx_b_r, int16_t *xp, const float *g2, const float *g4,
                        const float *g6, const float *g8, const float *g12, float *vp, float mass, float a_mid,
                        float dt, float *f2max, float vmax[3], double *ptotal);

/* PP short-range force and kick.  Replaces pp_force_kernel.cu:960-1050 and the
 * CPU pp_force_kernel.c:393-445 (bound at kick.f90:13-30).  ptotal: particles
 * kicked per subtile; ttotal: device seconds of the PP stage, reported on the
 * first subtile of each tile. */
void c_pp_force_kernel(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                       const int32_t *ratio_sf, int32_t *rhoc, int64_t *idx_b_r, int16_t *xp, float *vp,
                       float mass, float a_mid, float dt, float *f2max, float vmax[3], double *ptotal,
                       double *ttotal);

/* Release PM3 device state (pm3_fft_cuda.cu:621-628, finalize.f90:18-21). */
void c_pm3_fft_finalize(void);
/* Release PP / velocity device state (pp_force_kernel.cu:539-547). */
void c_gpu_velocity_finalize(void);

/* ---- status-returning variants (same arguments) ---- */
int cube_pm3_force(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf,
                   const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp, const float *const gk[5],
                   float *vp, float mass, float a_mid, float dt, float *f2max, float vmax[3], double *ptotal);
int cube_pp_force(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                  const int32_t *ratio_sf, const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp,
                  float *vp, float mass, float a_mid, float dt, float *f2max, float vmax[3], double *ptotal,
                  double *ttotal);

/* Whole fine-scale kick (PM3 then PP) with one upload of xp/rhoc/idx_b_r/vp
 * and one download of vp.  Equivalent to cube_pm3_force followed by
 * cube_pp_force (kick.f90:138-236).  out[0] = PM3 f2max, out[1] = PP f2max,
 * out[2..4] = vmax after the kick.  ptotal may be NULL. */
int cube_kick_fine(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                   const int32_t *ratio_sf, const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp,
                   const float *const gk[5], float *vp, float mass, float a_mid, float dt, float out[5],
                   double *ptotal);

/* Same kick on device-resident arrays; enqueued on `stream` (a cudaStream_t,
 * NULL = the library's stream) without host synchronisation.  d_out (6 words
 * of device memory) receives the 5 floats of cube_kick_fine and, in word 5,
 * an int32 mask of device-side failures (bit CUBE_ERR_CAPACITY or
 * CUBE_ERR_INVALID; 0 = none) when the stream reaches it.  The small host
 * tables are read during the call.  d_xp and d_vp may be NULL when n_used is 0
 * (an image without particles). */
int cube_kick_fine_device(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                          const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r,
                          const int16_t *d_xp, int64_t n_used, const float *const gk[5], float *d_vp, float mass,
                          float a_mid, float dt, float *d_out, void *stream);

/* ---- the device kick as one CUDA graph (no reference counterpart) ---- */

/* cube_kick_fine_device captured once as a CUDA graph and replayed per step, so that a
 * time loop pays one graph launch per kick.  Creation runs one kick on a scratch copy of
 * d_vp (d_vp itself is untouched) to size every buffer, then captures the kick on the
 * library's own stream.  The graph keeps the device pointers, n_used, the tables
 * (ires, ixyz3, apm3, ratio_sf) and mass/a_mid/dt of this call: a replay kicks the
 * current contents of these arrays, and a new graph is needed when the layout, the
 * subtile levels or n_used change.  Geometries CUBE_PM3_PERIODIC and
 * CUBE_PM3_TILE_PERIODIC only (CUBE_ERR_INVALID for CUBE_PM3_SUBTILE).  A replay must not
 * overlap another call of the library. */
typedef struct cube_kick_graph cube_kick_graph;
int cube_kick_graph_create(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                           const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r,
                           const int16_t *d_xp, int64_t n_used, float *d_vp, float mass, float a_mid, float dt,
                           float *d_out, cube_kick_graph **graph);
/* Enqueue one replay on `stream` (a cudaStream_t; NULL = the default stream). */
int cube_kick_graph_launch(cube_kick_graph *graph, void *stream);
int cube_kick_graph_destroy(cube_kick_graph *graph);

/* ---- PM1 and PM2, the long-range layers of the reference's force split ---- */

/* PM1 (kick.f90:61-73 with particle_mesh.f90, pm_layer 1): TSC deposit of the physical
 * particles on one periodic mesh of nc^3 coarse cells over the image (gridsize = ratio_cs),
 * the Green table Green_3D(nc, apm1c, 0, ratio_cs) of initialize.f90:129 (tabulated here in
 * FP64), the 4-point difference, and the TSC gather and kick of vp by a_mid dt / (6 pi) for the
 * physical particles.  Device arrays; the call waits for f2max and vmax.  nc a multiple of 4. */
int cube_pm1_force_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                          float *d_vp, float mass, float a_mid, float dt, float apm1c, float *f2max, float vmax[3],
                          void *stream);
/* PM2 (kick.f90:77-105, pm_thread of kick.f90:403-568 with pm_layer 2): per parent tile, the fine
 * mesh of the tile with its buffers (ngt = ngp + 2 ngb points per side, gridsize 1), every stored
 * copy of the tile deposited (nloop = ncb), Green_3D(ngt, apm2, apm1, 1) of initialize.f90:135,
 * and the kick of the tile's physical particles.  The tiles' meshes are transformed as one batch.
 * Same conventions as cube_pm1_force_device.  The range apm1 should not exceed the buffer depth
 * ngb, as in the reference (apm1 = 14, ngb = 16). */
int cube_pm2_force_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                          float *d_vp, float mass, float a_mid, float dt, float apm2, float apm1, float *f2max,
                          float vmax[3], void *stream);

/* ---- drift and buffer rebuild (drift.f90, buffer_grid.f90, buffer_particle.f90) ---- */

/* One drift of the configured image followed by the rebuild of its periodic buffers:
 * drift.f90:1-161 (new offsets xp + nint(dt_mid vp / (x_resolution ratio_cs)) with int16
 * wrap, re-binning by ceiling(x + dt_mid vp / ratio_cs), compaction; the order inside a
 * cell is the reference's layered visiting order with nlayer = 2 ceiling(dt_mid vz_max /
 * ratio_cs) + 2) and then buffer_grid + buffer_x + buffer_v (main.f90:27-31 without the
 * kick): every buffer cell receives the particles of the physical cell it mirrors, in
 * order.  With CUBE_PM3_TILE_PERIODIC each tile is its own periodic box.  Inputs and
 * outputs are distinct device arrays; pid (one int64 per stored copy) may be NULL.  The
 * call waits for the new sizes: *n_used_new receives the stored copies of the new image
 * (physical + buffers) and *n_physical (may be NULL) the physical particles.  Returns
 * CUBE_ERR_CAPACITY, with only rhoc_new and idx_b_r_new written, when *n_used_new >
 * cap_new; CUBE_ERR_INVALID for a non-finite nlayer or nint beyond the default integer. */
int cube_drift_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, const float *d_vp,
                      const int64_t *d_pid, int64_t n_used, float dt_mid, float vz_max, int32_t *d_rhoc_new,
                      int64_t *d_idx_b_r_new, int16_t *d_xp_new, float *d_vp_new, int64_t *d_pid_new,
                      int64_t cap_new, int64_t *n_used_new, int64_t *n_physical, void *stream);
/* Same on host arrays, in place (the reference's own arrays, `capacity` stored copies). */
int cube_drift(int32_t *rhoc, int64_t *idx_b_r, int16_t *xp, float *vp, int64_t *pid, int64_t n_used,
               int64_t capacity, float dt_mid, float vz_max, int64_t *n_used_new, int64_t *n_physical);
/* buffer_v (buffer_particle.f90:14-21): every buffer copy takes the velocity of the
 * physical particle it mirrors, in place on device arrays; enqueued on `stream`. */
int cube_buffer_v_device(const int32_t *d_rhoc, const int64_t *d_idx_b_r, float *d_vp, int64_t n_used,
                         void *stream);

/* ---- checkpoint files (checkpoint.f90, particle_initialization.f90) ---- */

/* sim_header of parameters.f90:141-164.  In the info file it is 13 int64 followed by 19
 * real(4), 180 bytes, no padding (a Fortran stream write of the derived type). */
typedef struct cube_sim_header {
  int64_t nplocal, npglobal, izipx, izipv, image, nn, nnt, nt, ncell, ncb, timestep, cur_checkpoint,
      cur_halofind;
  float a, t, tau, dt_pp, dt_pm3, dt_pm2, dt_pm1, dt_vmax, mass_p_cdm, box, h0, omega_m, omega_l, s8, vsim2phys,
      sigma_vres, sigma_vi, z_i, vz_max;
} cube_sim_header;

/* Write the checkpoint of the configured image (checkpoint.f90:11-38): files
 * prefix + {info, xp, vp, np, id} + suffix, as the reference names them
 * (basic_functions.f08:60-86: prefix "<opath>image<i>/<z>_", suffix "_<i>.bin").  The image
 * is given with its buffers; its physical particles are written tile by tile, row by row, the
 * order the reference's arrays hold right after a drift.  header->nplocal is set from the
 * image; pid NULL writes no id file.  Host arrays; needs no GPU. */
int cube_snapshot_write(const char *prefix, const char *suffix, const cube_sim_header *header, const int32_t *rhoc,
                        const int64_t *idx_b_r, const int16_t *xp, const float *vp, const int64_t *pid);
/* Read one (particle_initialization.f90:19-60): the header, the physical counts rhoc_phys
 * (C view [nnt^3][nt][nt][nt] of rhoc(1:nt,1:nt,1:nt,:,:,:); NULL skips them) and nplocal
 * particles into xp / vp / pid (pid NULL skips the id file).  CUBE_ERR_INVALID when the
 * stored formats (izipx, izipv = 2) or nnt / nt differ from the configured layout;
 * CUBE_ERR_CAPACITY, with the header filled, when nplocal > capacity.  The buffers are rebuilt
 * by a drift with dt_mid = 0 on the image of physical cells (cube_drift). */
int cube_snapshot_read(const char *prefix, const char *suffix, cube_sim_header *header, int32_t *rhoc_phys,
                       int16_t *xp, float *vp, int64_t *pid, int64_t capacity);

/* ---- CIC power spectrum (utilities/cicpower.f90, utilities/powerspectrum.f90) ---- */

/* CIC deposit of the image's physical particles on a cell-centred nw^3 grid
 * (cicpower.f90:55-70), delta = rho nw^3 / n_physical - 1, one R2C transform, and the
 * linear-k binning of powerspectrum.f90:52-94: for bins b = 0..nbin (nbin <= 0: nint(nw/2
 * sqrt 3)), bins[b] = modes, bins[nbin+1+b] = sum |k|, bins[2(nbin+1)+b] = sum |delta_k|^2 /
 * sinc^4 and bins[3(nbin+1)+b] = sum 4 pi |k|^3 |delta_k|^2 / sinc^4 (delta_k = FFT / nw^3,
 * |k| in grid units).  nw even, 2..2048.  Waits for the result (host array). */
int cube_power_spectrum(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                        int64_t n_physical, int32_t nw, int32_t nbin, double *bins, void *stream);

/* ---- FP64 conservation sums (no reference counterpart) ---- */

/* Momentum and kinetic-energy change of the physical particles (the interior coarse cells of
 * every tile) between two velocity arrays of the same device image, typically vp before and
 * after a kick: out[0..2] = sum m (vb - va) per axis, out[3] = sum m/2 (|vb|^2 - |va|^2),
 * out[4..6] = sum |m (vb - va)| per axis (the scale against which out[0..2] is measured),
 * out[7] = the number of physical particles.  Reduced in FP64 on the device; the call waits
 * for `stream`.  The reference prints sums of the same kind as its own invariants
 * ("sum of PM3 density", kick.f90:183; "sum of PP count", kick.f90:230). */
int cube_kick_sums(const int32_t *d_rhoc, const int64_t *d_idx_b_r, int64_t n_used, const float *d_va,
                   const float *d_vb, float mass, double out[8], void *stream);

/* ---- PP kernel shape autotuner (no reference counterpart) ---- */

/* The PP force kernel comes in several shapes: `chunk` i-particles per work item (a
 * crowded PP cell of n particles is split into ceil(n / chunk) items, one warp each),
 * `jtile` candidates a warp stages in shared memory between flushes, the pair loop
 * unrolled `unroll` times, registers budgeted for `blocks` resident blocks per SM, and
 * `packed` = 1 for the pair law on packed f32x2 arithmetic (two candidates per lane and
 * instruction; each pair's force is the scalar one bit for bit).  By
 * default the first PP kick of each (layout, per-tile PP grids, PP ranges, octave of
 * n_used) times every shape on its own particles (work list + force kernel, into scratch
 * velocities; the host waits for it once) and that key keeps the fastest; a kick being
 * captured into a graph that meets an untimed key uses shape 0.  Results of different
 * shapes differ only by FP32 summation order. */
typedef struct cube_pp_shape_info {
  int32_t chunk, jtile, unroll, blocks, packed;
  float ms; /* the last tuning's time of the shape (work list + force kernel), -1 if never timed */
} cube_pp_shape_info;
/* shape >= 0: use that shape for every PP kick; -1: autotune (default; forgets earlier picks). */
int cube_pp_set_shape(int32_t shape);
/* The shape table (up to `cap` entries), its size and the shape of the last PP kick. */
int cube_pp_shapes(cube_pp_shape_info *out, int32_t cap, int32_t *n_shapes, int32_t *current);
/* Inspection of the PP work list the last PP kick ran (waits for the device):
 * out[0] = work items, out[1] = items that hold one chunk of a PP cell split across
 * several items, out[2] = items that group two or four sparse PP cells along x,
 * out[3] = the largest particle count of one item.  All zero before the first kick. */
int cube_pp_work_stats(int64_t out[4]);

/* ---- learned PP shell (no reference counterpart) ---- */

/* A small MLP that predicts, per particle, the force that the cutoff-1 split (PM3
 * softened at 1 fine cell plus PP within 1 fine cell) misses against the cutoff-2 split,
 * from the CIC density of the image on the 4^3 fine cells around the particle (as
 * log(1 + rho)) and the particle's offset in its cell: 67 inputs (padded to 80, BF16),
 * layers 128, 128, 128 with tanh-GELU, 3 outputs; BF16 tensor-core GEMMs with FP32
 * accumulation.  Parameters (FP32, flat, CUBE_MLP_PARAMS floats): W1 [128][80], b1 [128],
 * W2 [128][128], b2 [128], W3 [128][128], b3 [128], W4 [3][128], b4 [3].  The single
 * periodic image geometry (CUBE_PM3_PERIODIC) only. */
#define CUBE_MLP_PARAMS 43779
#define CUBE_MLP_INPUTS 80
typedef struct cube_mlp cube_mlp;
/* Upload the parameters; training steps take at most batch_cap rows (a multiple of 16). */
int cube_mlp_create(const float *params, int32_t batch_cap, cube_mlp **mlp);
int cube_mlp_destroy(cube_mlp *mlp);
/* Current parameters and the gradients of the last training step (either may be NULL). */
int cube_mlp_get_params(cube_mlp *mlp, float *params, float *grads);
/* Input rows d_X (BF16 [n_used][80], zeros for buffer copies) of every stored copy of the
 * image, in storage order (the training input). */
int cube_mlp_features(const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp, int64_t n_used,
                      void *d_X, void *stream);
/* One Adam step (lr, betas 0.9 / 0.999, eps 1e-8) on the rows d_rows[0..batch) of d_X with
 * targets d_T [rows][3]: mean squared error, added to *d_loss. */
int cube_mlp_train_step(cube_mlp *mlp, const void *d_X, const float *d_T, const int32_t *d_rows, int32_t batch,
                        float lr, float *d_loss, void *stream);
/* Outputs d_Y [rows][3] of the rows of d_X. */
int cube_mlp_forward(cube_mlp *mlp, const void *d_X, int64_t rows, float *d_Y, void *stream);
/* vp += a_mid*dt/(6 pi) * scale * MLP(inputs) for the interior copies of the image
 * (inputs, density and network in one pass; the cutoff-1 kick itself is a separate call). */
int cube_mlp_kick(cube_mlp *mlp, const int32_t *d_rhoc, const int64_t *d_idx_b_r, const int16_t *d_xp,
                  int64_t n_used, float *d_vp, float scale, float a_mid, float dt, void *stream);

/* The learned shell's per-cell check and fallback.  d_vp_learned and d_vp_full hold the
 * velocities after the learned kick (cutoff-1 split plus cube_mlp_kick) and after the
 * full-cutoff kick (the plain cube_kick_fine_device) of the same image, both from d_vp0.  The
 * full-cutoff kick is the reference for the network: every coarse cell with physical particles
 * is checked on its first `samples` (1..32) particles in storage order, by the relative rms difference of
 * the two velocity changes there; a cell over `bound` takes the full-cutoff velocities for all
 * its particles, the others keep the learned ones.  d_vp_out (may be d_vp_learned) receives
 * the result.  out[0] = cells checked, out[1] = cells over the bound, out[2] = particles that
 * fell back, out[3] = relative rms of the learned change against the full-cutoff one over all
 * samples, out[4] = samples.  Waits for `stream`.  No reference counterpart. */
int cube_learned_fallback(const int32_t *d_rhoc, const int64_t *d_idx_b_r, int64_t n_used, const float *d_vp0,
                          const float *d_vp_learned, const float *d_vp_full, float bound, int32_t samples,
                          float *d_vp_out, double out[5], void *stream);

/* ---- allocation-free PP kick ---- */

/* Largest input cube_pp_force_noalloc accepts: stored particles (n_used) and
 * PP cells over all tiles (also the bound on coarse cells over all extended
 * tiles).  The scratch for this size is one static device array of about
 * 22 MB that every GPU loading the library holds until the process exits. */
#define CUBE_NOALLOC_MAX_PARTICLES 524288
#define CUBE_NOALLOC_MAX_CELLS 262144

/* The PP kick of cube_pp_force on device-resident arrays, for callers that
 * cannot let a library allocate device memory (their allocator owns every
 * byte, or an allocation-free execution policy is in force).  It calls no
 * cudaMalloc, cudaFree or other allocating routine: the caller passes the
 * inputs (d_rhoc, d_idx_b_r, d_xp) and outputs (d_vp is kicked in place;
 * d_out, 6 words of device memory, receives PP f2max in word 1, vmax in words
 * 2..4 and a device failure mask in word 5), and all scratch lives in a
 * file-scope device array.  Enqueued on `stream` (NULL = the default stream)
 * on the current device, without host synchronisation.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it; make that first call before any stream
 * capture begins.  Every call shares the array and
 * it keeps the previous call's contents (counters are reset by each call):
 * calls that overlap on the GPU race on it.  Returns CUBE_ERR_CAPACITY beyond
 * CUBE_NOALLOC_MAX_PARTICLES / CUBE_NOALLOC_MAX_CELLS, 64 tiles or 4096
 * subtiles.  This entry point has no counterpart in the reference. */
int cube_pp_force_noalloc(const int32_t *isort, const int32_t *ires, const int32_t *ixyz3, const float *apm3,
                          const int32_t *ratio_sf, const int32_t *d_rhoc, const int64_t *d_idx_b_r,
                          const int16_t *d_xp, int64_t n_used, float *d_vp, float mass, float a_mid, float dt,
                          float *d_out, void *stream);

/* ---- inspection (parity checks) ---- */

/* Binning of one parent tile as the PP pass builds it, in the reference's
 * conventions (pp_force_kernel.c:196-274): key of every sorted particle,
 * storage index ip (ip_local[values[]]) of every sorted particle, cell_start
 * (grid_num + 1 entries, tile-local), sorted positions xf [3][N].  Capacities
 * in elements; *n_out = N, *grid_out = grid_num.  Runs the binning on the
 * given host inputs.  spatial = 0 gives the reference's order inside each PP
 * cell (stable by storage slot); spatial = 1 gives the order the kick uses
 * (Morton sub-cell, then storage slot), with the same keys and cell_start. */
int cube_pp_bin_tile(const int32_t *ires, const int32_t *ixyz3, const int32_t *ratio_sf, const int32_t *rhoc,
                     const int64_t *idx_b_r, const int16_t *xp, int32_t tile, int32_t spatial, uint32_t *keys,
                     int64_t *ip, int32_t *cell_start, float *xf, int64_t cap_n, int64_t cap_grid, int64_t *n_out,
                     int64_t *grid_out);

/* Number of ordered PP pairs (i interior, 0 < r^2 < range^2) the kick evaluates
 * for these inputs -- the algorithmic work of pp_force_kernel.c:282-325, counted
 * by the same binning and work list on the device.  Host inputs as cube_pp_force. */
int cube_pp_pair_count(const int32_t *ires, const int32_t *ixyz3, const float *apm3, const int32_t *ratio_sf,
                       const int32_t *rhoc, const int64_t *idx_b_r, const int16_t *xp, int64_t *pairs);

/* Green table of the periodic mesh (FP64 tabulation on the device, Green.f90:1-80),
 * copied to host G[n][n][n/2+1]. */
int cube_green_table(int32_t n, float apm_soft, float apm_range, float gridsize, float *G);

/* FP64 periodic softened direct sum (Ewald split) on the device for nt targets:
 * pos [N][3] and targets are host arrays, F [nt][3] is written on the host.
 * Used to state force errors; not part of the kick. */
int cube_force_truth_fp64(const double *pos, int64_t n, double box, double app, const int64_t *targets, int64_t nt,
                          double alpha, double rcut, int32_t nmax, double *F);

/* Device time in ms of the last host-API kick's stages: [0] PM3 total,
 * [1] PP binning + work list, [2] PP force kernel, [3] whole device pipeline
 * (filled when timing is enabled).  In a kick with both parts the PP binning and
 * work list run beside PM3, so [0] + [1] + [2] can exceed [3]. */
int cube_stage_times(float ms[4]);
int cube_enable_timing(int on);
/* Stage times of every timed call since the previous read (oldest first, at
 * most max_calls, 4 floats per call as cube_stage_times); waits for them. */
int cube_timing_read(float *ms, int32_t max_calls, int32_t *n_calls);
/* Number of this library's own kernels enqueued so far (cuFFT's not included). */
int64_t cube_launch_count(void);
/* FP32 FMA throughput of this device in TFLOP/s, measured by a register-resident
 * FMA loop (the denominator of the PP kernel's roofline). */
int cube_fp32_peak_probe(float *tflops);

#ifdef __cplusplus
}
#endif
#endif /* CUBE2_B200_H */
