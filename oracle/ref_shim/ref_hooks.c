/*
 * ref_hooks.c — link-time hooks (-Wl,--wrap=...) around the unmodified
 * muMatScale reference, used to pin the oracle and to generate golden
 * vectors.  Test infrastructure only.
 *
 *  --wrap=doiteration          (calculate.c:193)  dump the subblock's fields
 *                               after chosen steps (MMSREF_DUMP_DIR,
 *                               MMSREF_DUMP_STEPS="a,b,c" or MMSREF_DUMP_EVERY=k);
 *                               with MMSREF_STEP_TIMES=<file>, rank 0 appends
 *                               "<timestep> <seconds>" after every step (the
 *                               halo exchanges keep the ranks in lockstep)
 *  --wrap=init_sb_nucleation   (grain.c:931)      optionally replace the
 *                               pre-drawn nucleation thresholds by a site file
 *                               (MMSREF_INJECT_SITES); dump the thresholds
 *                               that setup produced (MMSREF_DUMP_SETUP=1)
 *  --wrap=activateNewGrains    (grain.c:841)      optionally overwrite the
 *                               rotation matrix of new grains from a per-site
 *                               table (MMSREF_INJECT_ROT)
 *  --wrap=fs_change_diffuse    (growth.c:177)     with MMSREF_CURV=1 and
 *                               TipCurvature 1, call the reference's own
 *                               sb_curvature (curvature.c:31) first; the
 *                               reference defines it but never calls it.
 *
 * Dump file layout (little endian), one file per rank and step,
 * <dir>/r<rank>_s<timestep>.bin:
 *   char[8] "MMSDUMP1"; int64 rank, nproc, sbx, sby, sbz, gsdimx, gsdimy,
 *   gsdimz, timestep, num_grains, maxTotalGrains, gindex;
 *   f64 ce[N], cl[N], fs[N], d[N]; f64 dc[3N] (x,y,z packed per cell);
 *   i32 gr[N]; f32 nuc_threshold[N]; f64 temperature[N]; i32 ogr[N];
 *   grain_t grain_cache[num_grains] (136-byte records, globals.h:244)
 * with N = (gsdimx+2)(gsdimy+2)(gsdimz+2) in the reference's halo'd order.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "globals.h"
#include "functions.h"

extern SB_struct *lsp;
extern grain_t *grain_cache;

void __real_doiteration(void);
void __real_init_sb_nucleation(SB_struct *sb);
void __real_activateNewGrains(void);
void __real_fs_change_diffuse(SB_struct *lsp, void *unused);
void sb_curvature(void *vlsp, void *unused);

static long total_cells(void)
{
    return (long)(bp->gsdimx + 2) * (bp->gsdimy + 2) * (bp->gsdimz + 2);
}

static int step_wanted(uint64_t ts)
{
    const char *every = getenv("MMSREF_DUMP_EVERY");
    if (every && atol(every) > 0 && ts % (uint64_t)atol(every) == 0) return 1;
    const char *steps = getenv("MMSREF_DUMP_STEPS");
    if (!steps) return 0;
    const char *p = steps;
    while (*p) {
        char *end;
        unsigned long long v = strtoull(p, &end, 10);
        if (end == p) break;
        if (v == ts) return 1;
        p = (*end == ',') ? end + 1 : end;
    }
    return 0;
}

static void write_dump(const char *tag)
{
    const char *dir = getenv("MMSREF_DUMP_DIR");
    if (!dir) return;
    char path[1024];
    snprintf(path, sizeof path, "%s/r%d_%s.bin", dir, iproc, tag);
    FILE *f = fopen(path, "wb");
    if (!f) {
        perror(path);
        exit(3);
    }
    long N = total_cells();
    int64_t hdr[12] = {iproc, nproc, lsp->coords.x, lsp->coords.y, lsp->coords.z,
                       bp->gsdimx, bp->gsdimy, bp->gsdimz, (int64_t)bp->timestep,
                       bp->num_grains, (int64_t)bp->maxTotalGrains, lsp->gindex};
    fwrite("MMSDUMP1", 1, 8, f);
    fwrite(hdr, sizeof hdr, 1, f);
    fwrite(lsp->ce, sizeof(double), N, f);
    fwrite(lsp->cl, sizeof(double), N, f);
    fwrite(lsp->fs, sizeof(double), N, f);
    fwrite(lsp->d, sizeof(double), N, f);
    fwrite(lsp->dc, sizeof(decentered_t), N, f);
    fwrite(lsp->gr, sizeof(int), N, f);
    fwrite(lsp->nuc_threshold, sizeof(float), N, f);
    fwrite(lsp->temperature, sizeof(double), N, f);
    fwrite(lsp->ogr, sizeof(int), N, f);
    fwrite(grain_cache, sizeof(grain_t), bp->num_grains, f);
    fclose(f);
}

double MPI_Wtime(void);

void __wrap_doiteration(void)
{
    __real_doiteration();
    static FILE *tf = NULL;
    static int tf_checked = 0;
    if (!tf_checked) {
        tf_checked = 1;
        const char *path = getenv("MMSREF_STEP_TIMES");
        if (path && iproc == 0) tf = fopen(path, "w");
    }
    if (tf) {
        fprintf(tf, "%llu %.9f\n", (unsigned long long)bp->timestep, MPI_Wtime());
        fflush(tf);
    }
    if (step_wanted(bp->timestep)) {
        char tag[64];
        snprintf(tag, sizeof tag, "s%llu", (unsigned long long)bp->timestep);
        write_dump(tag);
    }
}

typedef struct {
    int32_t gx, gy, gz;
    float threshold;
} inj_site;

void __wrap_init_sb_nucleation(SB_struct *sb)
{
    const char *path = getenv("MMSREF_INJECT_SITES");
    if (!path) {
        __real_init_sb_nucleation(sb);
    } else {
        FILE *f = fopen(path, "rb");
        if (!f) {
            perror(path);
            exit(3);
        }
        int64_t n = 0;
        if (fread(&n, sizeof n, 1, f) != 1) exit(3);
        for (int64_t s = 0; s < n; s++) {
            inj_site site;
            if (fread(&site, sizeof site, 1, f) != 1) exit(3);
            int lx = site.gx - (int)sb->coords.x * bp->gsdimx;
            int ly = site.gy - (int)sb->coords.y * bp->gsdimy;
            int lz = site.gz - (int)sb->coords.z * bp->gsdimz;
            if (lx < 0 || ly < 0 || lz < 0 || lx >= bp->gsdimx || ly >= bp->gsdimy ||
                lz >= bp->gsdimz)
                continue;
            long idx = SBIDX(lx + 1, ly + 1, lz + 1);
            if (!sb->mold[idx]) sb->nuc_threshold[idx] = site.threshold;
        }
        fclose(f);
    }
    const char *ds = getenv("MMSREF_DUMP_SETUP");
    if (ds && atoi(ds)) write_dump("setup");
}

typedef struct {
    int32_t gx, gy, gz, pad;
    double rotmat[9];
} inj_rot;

static inj_rot *g_rot = NULL;
static int64_t g_nrot = -1;

static void load_rot(void)
{
    g_nrot = 0;
    const char *path = getenv("MMSREF_INJECT_ROT");
    if (!path) return;
    FILE *f = fopen(path, "rb");
    if (!f) {
        perror(path);
        exit(3);
    }
    if (fread(&g_nrot, sizeof g_nrot, 1, f) != 1) exit(3);
    g_rot = (inj_rot *)malloc(sizeof(inj_rot) * (size_t)(g_nrot ? g_nrot : 1));
    if (fread(g_rot, sizeof(inj_rot), (size_t)g_nrot, f) != (size_t)g_nrot) exit(3);
    fclose(f);
}

void __wrap_activateNewGrains(void)
{
    if (g_nrot < 0) load_rot();
    int before = bp->num_grains;
    __real_activateNewGrains();
    if (g_nrot <= 0) return;
    for (int id = before; id < bp->num_grains; id++) {
        grain_t *g = &grain_cache[id];
        size_t cx, cy, cz;
        realcoord2scoord(g->nuc_x, g->nuc_y, g->nuc_z, &cx, &cy, &cz);
        for (int64_t s = 0; s < g_nrot; s++) {
            if (g_rot[s].gx == (int32_t)cx && g_rot[s].gy == (int32_t)cy &&
                g_rot[s].gz == (int32_t)cz) {
                memcpy(&g->rotmat[0][0], g_rot[s].rotmat, sizeof(double) * 9);
                break;
            }
        }
    }
}

void __wrap_fs_change_diffuse(SB_struct *sb, void *unused)
{
    const char *c = getenv("MMSREF_CURV");
    if (c && atoi(c) && bp->tip_curv) sb_curvature(sb, NULL);
    __real_fs_change_diffuse(sb, unused);
}
