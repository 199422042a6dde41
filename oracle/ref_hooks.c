/*
 * Test infrastructure only (oracle): allocation recorders linked into the
 * reference build of pp_force_kernel.c (see ref_hooks.h and build_ref.py).
 *
 * c_pp_force_kernel_tile (pp_force_kernel.c:134-391) allocates, in this order:
 *   seq 0  _xf        (:182)   seq 1 _vf (:183)   seq 2 _af (:187, [3][nptile])
 *   seq 3  ip_local   (:188)   seq 4 keys (:193)  seq 5 values (:194)
 *   seq 6,7 radix scratch (:77-78, freed inside radix_sort_u32_pair)
 *   seq 8  _xf_sorted (:246, [3][N])   seq 9 cell_start (:259, grid_num+1)
 * and frees ip_local last (:378).  When capture is switched on, the recorder
 * copies the contents of seq 2,3,4,5,8,9 at the moment the reference frees
 * them, i.e. after the sort, the cell_start fill-in and the force/velocity
 * update.  Capture is only meaningful for one serial call of
 * c_pp_force_kernel_tile; with capture off the recorders only forward to libc.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#undef malloc
#undef free

#define CUBE_REF_SLOTS 10

static int g_capture = 0;
static int g_seq = 0;
static struct {
  void *ptr;
  size_t size;
} g_live[CUBE_REF_SLOTS];
static struct {
  void *data;
  size_t size;
} g_snap[CUBE_REF_SLOTS];

void *cube_ref_malloc(size_t n) {
  void *p = malloc(n ? n : 1);
  if (g_capture && g_seq < CUBE_REF_SLOTS) {
    g_live[g_seq].ptr = p;
    g_live[g_seq].size = n;
  }
  if (g_capture) g_seq++;
  return p;
}

void cube_ref_free(void *p) {
  if (g_capture && p) {
    for (int s = 0; s < CUBE_REF_SLOTS; s++) {
      if (g_live[s].ptr == p) {
        if (s == 2 || s == 3 || s == 4 || s == 5 || s == 8 || s == 9) {
          free(g_snap[s].data);
          g_snap[s].data = malloc(g_live[s].size ? g_live[s].size : 1);
          g_snap[s].size = g_live[s].size;
          memcpy(g_snap[s].data, p, g_live[s].size);
        }
        g_live[s].ptr = NULL;
        if (s == 3) g_seq = 0; /* ip_local is the last buffer the tile frees */
        break;
      }
    }
  }
  free(p);
}

/* Switch capture on (1) or off (0); switching on clears earlier snapshots. */
void cube_ref_capture(int on) {
  g_capture = on;
  g_seq = 0;
  for (int s = 0; s < CUBE_REF_SLOTS; s++) {
    g_live[s].ptr = NULL;
    free(g_snap[s].data);
    g_snap[s].data = NULL;
    g_snap[s].size = 0;
  }
}

/* Size in bytes of snapshot `slot` (0 if none). */
size_t cube_ref_snapshot_size(int slot) {
  if (slot < 0 || slot >= CUBE_REF_SLOTS) return 0;
  return g_snap[slot].size;
}

/* Copy snapshot `slot` into dst (at most cap bytes); returns bytes copied. */
size_t cube_ref_snapshot_copy(int slot, void *dst, size_t cap) {
  if (slot < 0 || slot >= CUBE_REF_SLOTS || !g_snap[slot].data) return 0;
  size_t n = g_snap[slot].size < cap ? g_snap[slot].size : cap;
  memcpy(dst, g_snap[slot].data, n);
  return n;
}
