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
 *  --wrap=loop                 (loop.c:186)       with
 *                               MMSREF_INJECT_SUBSTRATE=<file>, pre-fill a
 *                               substrate of grains before the first step, as
 *                               mms_set_grains plus a gr/fs upload does on the
 *                               device: grains 1..n get the file's rotation
 *                               matrices (num_grains = n + 1, so nucleated
 *                               grains continue from n + 1), and interior
 *                               planes 1..top of every column (x, y) take the
 *                               column's grain id with fs = 1.  File: int32
 *                               gx, gy, top, n; int32 col[gy][gx] (grain id of
 *                               each column, 0 = none); f64 rot[n][9].
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
void __real_loop(uint64_t restart, double gStartTime);
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

void __wrap_loop(uint64_t restart, double gStartTime)
{
    const char *path = getenv("MMSREF_INJECT_SUBSTRATE");
    if (path && !restart) {
        FILE *f = fopen(path, "rb");
        if (!f) {
            perror(path);
            exit(3);
        }
        int32_t hdr[4];
        if (fread(hdr, sizeof(int32_t), 4, f) != 4) exit(3);
        const int gx = hdr[0], gy = hdr[1], top = hdr[2], n = hdr[3];
        if (gx != bp->gnsbx * bp->gsdimx || gy != bp->gnsby * bp->gsdimy || n < 0 ||
            (uint64_t)n + 1 > bp->maxTotalGrains + 1) {
            fprintf(stderr, "%s: substrate does not fit this deck\n", path);
            exit(3);
        }
        int32_t *col = (int32_t *)malloc(sizeof(int32_t) * (size_t)gx * gy);
        double *rot = (double *)malloc(sizeof(double) * 9 * (size_t)(n ? n : 1));
        if (fread(col, sizeof(int32_t), (size_t)gx * gy, f) != (size_t)gx * gy ||
            fread(rot, sizeof(double), 9 * (size_t)n, f) != 9 * (size_t)n)
            exit(3);
        fclose(f);
        for (int g = 0; g < n; g++) {
            memset(&grain_cache[g + 1], 0, sizeof(grain_t));
            memcpy(&grain_cache[g + 1].rotmat[0][0], rot + 9 * (size_t)g, sizeof(double) * 9);
        }
        bp->num_grains = n + 1;
        for (int k = 1; k <= bp->gsdimz; k++) {
            const int K = (int)lsp->coords.z * bp->gsdimz + k;  /* global interior plane, 1-based */
            if (K > top) continue;
            for (int j = 1; j <= bp->gsdimy; j++)
                for (int i = 1; i <= bp->gsdimx; i++) {
                    const int X = (int)lsp->coords.x * bp->gsdimx + i - 1;
                    const int Y = (int)lsp->coords.y * bp->gsdimy + j - 1;
                    const int id = col[(size_t)Y * gx + X];
                    if (id <= 0) continue;
                    const long idx = SBIDX(i, j, k);
                    lsp->gr[idx] = id;
                    lsp->fs[idx] = 1.0;
                }
        }
        free(col);
        free(rot);
    }
    __real_loop(restart, gStartTime);
}
