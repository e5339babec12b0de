/*
 * mms_oracle.h — CPU restatement of the muMatScale CA step, used ONLY as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.
 * It is never linked into, imported by, or called from the product.
 *
 * One domain on the reference's halo'd global grid, with the per-rank
 * orderings of an NSubblocks MPI run emulated (rand() streams, grain ids,
 * interface-list slots).  Every function follows the reference file:line it
 * cites in mms_oracle.c.
 */
#ifndef MMS_ORACLE_H
#define MMS_ORACLE_H

#include <stdint.h>
#include "../include/mms.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mmso mmso;

mmso *mmso_create(const mms_params *p, int *status);
void mmso_destroy(mmso *o);
int mmso_set_sites(mmso *o, int64_t n, const int32_t *gxyz, const float *thr);
int mmso_set_site_orientations(mmso *o, int64_t n, const int32_t *gxyz, const double *rot9);
int mmso_set_grains(mmso *o, int n, const double *rot9);
int mmso_set_field(mmso *o, int field, const void *in);
/* enable the sb_curvature call before fs_change when TipCurvature is 1 */
void mmso_enable_curvature(mmso *o, int on);
int mmso_step(mmso *o, int nsteps);
uint64_t mmso_timestep(const mmso *o);
int mmso_num_grains(const mmso *o);
size_t mmso_num_cells(const mmso *o);
int mmso_get_field(mmso *o, int field, void *out);
double mmso_reduce(mmso *o, int what);
void mmso_get_grains(mmso *o, int first, int count, mms_grain *out);
void mmso_grain_summary(mmso *o, mms_grain_summary *s);
int mmso_run(mmso *o, int verbose);
/* the reference XDMF writer's grain renumbering on rank 0's stream */
int mmso_xdmf_renumber(mmso *o, uint64_t *out, int cap);
/* glibc rand() replay check: n values of srand(seed) + rand() */
void mmso_rand_sequence(unsigned seed, int n, int32_t *out);

#ifdef __cplusplus
}
#endif
#endif
