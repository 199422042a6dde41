/*
 * Test infrastructure only (oracle).  Force-included (-include) in front of the
 * reference's pp_force_kernel.c when oracle/build_ref.py compiles it.  It
 * renames the reference's malloc/free calls to the recorders in ref_hooks.c so
 * that the arrays the reference builds inside c_pp_force_kernel_tile (cell keys,
 * sort values, cell_start, sorted positions, ip_local, forces) can be copied
 * out just before the reference frees them.  Nothing in the reference's
 * arithmetic changes; the recorders pass every call through to libc.
 */
#ifndef CUBE_REF_HOOKS_H
#define CUBE_REF_HOOKS_H
#include <stdlib.h>
#include <stddef.h>
void *cube_ref_malloc(size_t n);
void cube_ref_free(void *p);
#define malloc cube_ref_malloc
#define free cube_ref_free
#endif
